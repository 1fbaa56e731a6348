// The C ABI (include/omega_h.h, include/omega_h_b200.h) over the device mesh.
// Every entry point converts C++ failures into an error code readable with
// osh_b200_last_error() and returns 0 / NULL instead of aborting.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <exception>

#include "../../include/omega_h.h"
#include "../../include/omega_h_b200.h"
#include "batch.hpp"
#include "fields.hpp"
#include "serve.hpp"
#include "passes.hpp"
#include "vtk_io.hpp"

using osh::Failure;
using osh::Mesh;
using osh::u32;
using osh::u64;

namespace osh {
void swap_table_host(u32 rs, u32* ntri, u32* nmesh, u32* nint, u32* tris, u32* iedges);
}

#define M(h) reinterpret_cast<Mesh*>(h)

#define API_TRY try {
#define API_CATCH(ret)                                   \
  }                                                      \
  catch (Failure const& f)                               \
  {                                                      \
    osh::set_error(f.code, f.what());                    \
    return ret;                                          \
  }                                                      \
  catch (std::exception const& e)                        \
  {                                                      \
    osh::set_error(osh::E_CUDA, e.what());               \
    return ret;                                          \
  }

#define API_CATCH_VOID                                   \
  }                                                      \
  catch (Failure const& f)                               \
  {                                                      \
    osh::set_error(f.code, f.what());                    \
    return;                                              \
  }                                                      \
  catch (std::exception const& e)                        \
  {                                                      \
    osh::set_error(osh::E_CUDA, e.what());               \
    return;                                              \
  }

using osh::launch_kernel;
using osh::pdl_wait;

namespace {

void need(bool ok, char const* what)
{
  if (!ok) throw Failure(osh::E_ARG, what);
}

void sync(Mesh* m)
{
  osh::stream_sync(m->s);
  osh::check_device_timeouts(m->s);
}

// An array just allocated on m's stream, made ready for the caller's copies
// (osh_b200_copy_to_device runs on the legacy default stream, which waits
// for the legacy stream and for blocking streams, not for a non-blocking
// one): a wait only when m's stream is non-blocking; no kernel ran, so no
// timeout to check.
void ready_for_copies(Mesh* m)
{
  unsigned flags = 0;
  if (m->s) CK(cudaStreamGetFlags(m->s, &flags));
  if (flags & cudaStreamNonBlocking) osh::stream_sync(m->s);
}

__global__ void k_mark_classified(u32 n, u32 const* __restrict__ cd,
    u32 const* __restrict__ cid, u32 target_dim, u32 target_id, u32* __restrict__ marked)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // mark_class_kern + mark_or_kern (mark.cpp:149-167, omega_h.cpp:890-896)
  if (cd[i] == target_dim && (target_id == osh::INV || cid[i] == target_id)) marked[i] = 1;
}

// vert_identity_size (size.cpp:90-108)
__global__ void k_identity_size(u32 nv, u32 const* __restrict__ offs,
    u32 const* __restrict__ adj, double const* __restrict__ x, double* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  double xi[3];
  osh::load3(x, i, xi);
  double mx = 0;
  for (u32 j = offs[i]; j < offs[i + 1]; ++j) {
    double xo[3];
    osh::load3(x, adj[j], xo);
    double l = sqrt(osh::sqdist3(xo, xi));
    if (l > mx) mx = l;
  }
  out[i] = mx;
}

osh::Tag* tag_at(Mesh* m, u32 dim, u32 i)
{
  need(dim <= m->dim && i < m->tags[dim].size(), "tag index out of range");
  return &m->tags[dim][i];
}

}  // namespace

namespace {
template <class T>
struct DevOut {
  T* d;
  T* host;
  size_t n;
  cudaStream_t s;
  DevOut(T* h, size_t count, cudaStream_t st) : d(osh::dalloc<T>(count, st)), host(h), n(count), s(st) {}
  void back() { CK(cudaMemcpyAsync(host, d, n * sizeof(T), cudaMemcpyDeviceToHost, s)); }
  ~DevOut() { cudaFreeAsync(d, s); }
};
}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// omega_h.h

void osh_init(int*, char***)
{
  API_TRY
  int n = 0;
  CK(cudaGetDeviceCount(&n));
  need(n > 0, "no CUDA device");
  API_CATCH_VOID
}

void osh_fini(void) {}

void osh_free(osh_t h)
{
  API_TRY
  delete M(h);
  API_CATCH_VOID
}

osh_t osh_read_vtk(char const* filename)
{
  API_TRY
  need(filename != nullptr, "filename is NULL");
  return reinterpret_cast<osh_t>(osh::read_vtk(filename));
  API_CATCH(nullptr)
}

void osh_write_vtk(osh_t h, char const* filename)
{
  API_TRY
  need(h != nullptr && filename != nullptr, "mesh or filename is NULL");
  osh::write_vtk(*M(h), filename, false, false);
  API_CATCH_VOID
}

osh_t osh_new(unsigned elem_dim)
{
  API_TRY
  need(elem_dim >= 1 && elem_dim <= 3, "elem_dim must be 1, 2 or 3");
  return reinterpret_cast<osh_t>(new Mesh(elem_dim, true, true, nullptr));
  API_CATCH(nullptr)
}

unsigned* osh_build_ents(osh_t h, unsigned ent_dim, unsigned nents)
{
  API_TRY
  Mesh* m = M(h);
  need(ent_dim <= m->dim, "entity dimension above the mesh dimension");
  u32 vpe = ent_dim ? osh::deg(ent_dim, 0) : 0;
  u32* conn = osh::dalloc<u32>((size_t)nents * vpe, m->s);
  osh::dev_free(m->down[ent_dim][0], m->s);
  m->set_ents(ent_dim, nents, conn);
  ready_for_copies(m);
  return conn;
  API_CATCH(nullptr)
}

unsigned osh_dim(osh_t h) { return M(h)->dim; }

unsigned osh_nelems(osh_t h)
{
  API_TRY
  return M(h)->count(M(h)->dim);
  API_CATCH(0)
}

unsigned osh_nverts(osh_t h) { return M(h)->counts[0]; }

unsigned osh_count(osh_t h, unsigned dim)
{
  API_TRY
  return M(h)->count(dim);
  API_CATCH(0)
}

unsigned const* osh_down(osh_t h, unsigned high, unsigned low)
{
  API_TRY
  Mesh* m = M(h);
  need(low <= high && high <= m->dim, "bad dimensions");
  u32 const* r = m->ask_down(high, low);
  sync(m);
  return r;
  API_CATCH(nullptr)
}

unsigned const* osh_up(osh_t h, unsigned low, unsigned high)
{
  API_TRY
  Mesh* m = M(h);
  need(low <= high && high <= m->dim, "bad dimensions");
  u32 const* r = m->ask_up(low, high).adj;
  sync(m);
  return r;
  API_CATCH(nullptr)
}

unsigned const* osh_up_offs(osh_t h, unsigned low, unsigned high)
{
  API_TRY
  Mesh* m = M(h);
  need(low <= high && high <= m->dim, "bad dimensions");
  u32 const* r = m->ask_up(low, high).offs;
  sync(m);
  return r;
  API_CATCH(nullptr)
}

unsigned const* osh_up_dirs(osh_t h, unsigned low, unsigned high)
{
  API_TRY
  Mesh* m = M(h);
  need(low <= high && high <= m->dim, "bad dimensions");
  u32 const* r = m->ask_up(low, high).dirs;
  sync(m);
  return r;
  API_CATCH(nullptr)
}

unsigned const* osh_star(osh_t h, unsigned low, unsigned high)
{
  API_TRY
  Mesh* m = M(h);
  need(low <= high && high <= m->dim, "bad dimensions");
  u32 const* r = m->ask_star(low, high).adj;
  sync(m);
  return r;
  API_CATCH(nullptr)
}

unsigned const* osh_star_offs(osh_t h, unsigned low, unsigned high)
{
  API_TRY
  Mesh* m = M(h);
  need(low <= high && high <= m->dim, "bad dimensions");
  u32 const* r = m->ask_star(low, high).offs;
  sync(m);
  return r;
  API_CATCH(nullptr)
}

double const* osh_coords(osh_t h)
{
  API_TRY
  return M(h)->coords();
  API_CATCH(nullptr)
}

unsigned const* osh_own_rank(osh_t h, unsigned dim)
{
  API_TRY
  Mesh* m = M(h);
  need(dim <= m->dim, "bad dimension");
  if (!m->has_own_ranks(dim)) {
    if (m->parallel) {
      // mesh_ask_own_ranks (parallel_mesh.cpp:77-84) derives ranks and ids
      m->note_exchange(dim);
    } else {
      m->ranks_zero[dim] = true;
    }
  }
  u32 const* r = m->ask_own_ranks(dim);
  sync(m);
  return r;
  API_CATCH(nullptr)
}

unsigned const* osh_own_id(osh_t h, unsigned dim)
{
  API_TRY
  Mesh* m = M(h);
  need(dim <= m->dim, "bad dimension");
  if (!m->has_own_ids(dim)) m->ids_iota[dim] = true;
  u32 const* r = m->ask_own_ids(dim);
  sync(m);
  return r;
  API_CATCH(nullptr)
}

unsigned long const* osh_global(osh_t h, unsigned dim)
{
  API_TRY
  Mesh* m = M(h);
  need(dim <= m->dim, "bad dimension");
  u64 const* g = m->ask_globals(dim);
  if (g) sync(m);
  return reinterpret_cast<unsigned long const*>(g);
  API_CATCH(nullptr)
}

double* osh_new_field(osh_t h, unsigned dim, char const* name, unsigned ncomps,
    enum osh_transfer tt)
{
  API_TRY
  Mesh* m = M(h);
  need(dim <= m->dim && name, "bad field");
  if (osh::Tag* t = m->find_tag(dim, name)) return static_cast<double*>(t->data);
  double* d = osh::dalloc<double>((size_t)m->count(dim) * ncomps, m->s);
  m->add_tag(dim, osh::T_F64, name, ncomps, (u32)tt, d);
  ready_for_copies(m);
  return d;
  API_CATCH(nullptr)
}

double* osh_get_field(osh_t h, unsigned dim, char const* name)
{
  API_TRY
  osh::Tag* t = M(h)->find_tag(dim, name);
  need(t != nullptr, "no such field");
  return static_cast<double*>(t->data);
  API_CATCH(nullptr)
}

void osh_free_field(osh_t h, unsigned dim, char const* name)
{
  API_TRY
  M(h)->remove_tag(dim, name);
  API_CATCH_VOID
}

unsigned osh_nfields(osh_t h, unsigned dim)
{
  u32 n = 0;
  for (auto const& t : M(h)->tags[dim])
    if (t.type == osh::T_F64) ++n;
  return n;
}

char const* osh_field(osh_t h, unsigned dim, unsigned i)
{
  u32 n = 0;
  for (auto const& t : M(h)->tags[dim])
    if (t.type == osh::T_F64 && i == n++) return t.name.c_str();
  return nullptr;
}

unsigned osh_components(osh_t h, unsigned dim, char const* name)
{
  API_TRY
  osh::Tag* t = M(h)->find_tag(dim, name);
  need(t != nullptr, "no such field or label");
  return t->ncomps;
  API_CATCH(0)
}

unsigned* osh_new_label(osh_t h, unsigned dim, char const* name, unsigned ncomps)
{
  API_TRY
  Mesh* m = M(h);
  need(dim <= m->dim && name, "bad label");
  if (osh::Tag* t = m->find_tag(dim, name)) return static_cast<u32*>(t->data);
  u32* d = osh::dalloc<u32>((size_t)m->count(dim) * ncomps, m->s);
  m->add_tag(dim, osh::T_U32, name, ncomps, osh::X_NOT, d);
  ready_for_copies(m);
  return d;
  API_CATCH(nullptr)
}

unsigned* osh_get_label(osh_t h, unsigned dim, char const* name)
{
  API_TRY
  osh::Tag* t = M(h)->find_tag(dim, name);
  need(t != nullptr, "no such label");
  return static_cast<u32*>(t->data);
  API_CATCH(nullptr)
}

void osh_free_label(osh_t h, unsigned dim, char const* name)
{
  API_TRY
  M(h)->remove_tag(dim, name);
  API_CATCH_VOID
}

unsigned long* osh_new_global(osh_t h, unsigned dim)
{
  API_TRY
  Mesh* m = M(h);
  need(dim <= m->dim, "bad dimension");
  u64* g = osh::dalloc<u64>(m->count(dim), m->s);
  m->set_globals(dim, g);
  sync(m);
  return g;
  API_CATCH(nullptr)
}

void osh_accumulate_to_owner(osh_t, unsigned, char const*) {}
void osh_conform(osh_t, unsigned, char const*) {}

void osh_mark_classified(osh_t h, unsigned ent_dim, unsigned class_dim, unsigned class_id,
    unsigned* marked)
{
  API_TRY
  Mesh* m = M(h);
  osh::Tag* cd = m->find_tag(ent_dim, "class_dim");
  need(cd != nullptr, "no class_dim label");
  osh::Tag* ci = m->find_tag(ent_dim, "class_id");
  need(class_id == osh::INV || ci != nullptr, "no class_id label");
  u32 n = m->count(ent_dim);
  if (n) {
    CK(launch_kernel(k_mark_classified, dim3(osh::grid_for(n)), dim3(osh::BLOCK), 0, m->s, n,
        static_cast<u32 const*>(cd->data), ci ? static_cast<u32 const*>(ci->data) : nullptr,
        class_dim, class_id, marked));
    CK_LAUNCH();
  }
  sync(m);
  API_CATCH_VOID
}

// mesh_ensure_ghosting (omega_h.cpp:944-947): on one rank the entities stay
// as they are; the layer count and the owner caches change as the
// reference's do
void osh_ghost(osh_t h, unsigned nlayers)
{
  API_TRY
  Mesh* m = M(h);
  need(m->parallel || nlayers == 0, "ghosting needs a parallel mesh");
  m->ensure_ghosting(nlayers);
  sync(m);
  API_CATCH_VOID
}

// mesh_ghost_layers (parallel_mesh.cpp:175-180): 0 for a serial mesh
unsigned osh_num_ghost_layers(osh_t h) { return M(h)->parallel ? M(h)->ghost_layers : 0; }

unsigned osh_adapt(osh_t h, double size_ratio_floor, double good_element_quality,
    unsigned nsliver_layers, unsigned max_passes)
{
  API_TRY
  u32 r = osh::mesh_adapt(*M(h), size_ratio_floor, good_element_quality, nsliver_layers,
      max_passes);
  sync(M(h));
  return r;
  API_CATCH(0)
}

void osh_identity_size(osh_t h, char const* name)
{
  API_TRY
  Mesh* m = M(h);
  u32 nv = m->count(0);
  osh::Graph const& g = m->ask_star(0, 1);
  double* out = osh::dalloc<double>(nv, m->s);
  if (nv) {
    CK(launch_kernel(k_identity_size, dim3(osh::grid_for(nv)), dim3(osh::BLOCK), 0, m->s, nv, g.offs, g.adj,
        m->coords(), out));
    CK_LAUNCH();
  }
  m->add_tag(0, osh::T_F64, name, 1, osh::X_NOT, out);
  sync(m);
  API_CATCH_VOID
}

// ---------------------------------------------------------------------------
// omega_h_b200.h

int osh_b200_last_error(void) { return osh::last_error(); }
char const* osh_b200_last_error_message(void) { return osh::last_error_message(); }
void osh_b200_clear_error(void) { osh::clear_error(); }

unsigned osh_b200_refine_by_size(osh_t h, double qf)
{
  API_TRY
  u32 r = osh::refine_by_size(*M(h), qf);
  sync(M(h));
  return r;
  API_CATCH(0)
}

void osh_b200_uniformly_refine(osh_t h)
{
  API_TRY
  osh::uniformly_refine(*M(h));
  sync(M(h));
  API_CATCH_VOID
}

unsigned osh_b200_coarsen_by_size(osh_t h, double qf, double sf)
{
  API_TRY
  u32 r = osh::coarsen_by_size(*M(h), qf, sf);
  sync(M(h));
  return r;
  API_CATCH(0)
}

unsigned osh_b200_coarsen_slivers(osh_t h, double qf, unsigned nl)
{
  API_TRY
  u32 r = osh::coarsen_slivers(*M(h), qf, nl);
  sync(M(h));
  return r;
  API_CATCH(0)
}

unsigned osh_b200_swap_slivers(osh_t h, double gq, unsigned nl)
{
  API_TRY
  u32 r = osh::swap_slivers(*M(h), gq, nl);
  sync(M(h));
  return r;
  API_CATCH(0)
}

unsigned osh_b200_mesh_adapt(osh_t h, double sf, double gq, unsigned nl, unsigned mo)
{
  return osh_adapt(h, sf, gq, nl, mo);
}

static thread_local std::vector<osh::BatchMeshResult> t_batch_res;

int osh_b200_adapt_batch(osh_t* meshes, unsigned n, double sf, double gq, unsigned nl,
    unsigned mo, unsigned long long max_union_elems, unsigned* changed, int* status)
{
  API_TRY
  need(meshes != nullptr || n == 0, "meshes is NULL");
  std::vector<Mesh*> ms(n);
  for (unsigned i = 0; i < n; ++i) {
    need(meshes[i] != nullptr, "a mesh handle is NULL");
    ms[i] = M(meshes[i]);
  }
  t_batch_res.clear();
  if (n) osh::adapt_batch(ms, sf, gq, nl, mo, max_union_elems, t_batch_res);
  for (unsigned i = 0; i < n; ++i) {
    if (changed) changed[i] = t_batch_res[i].changed;
    if (status) status[i] = t_batch_res[i].status;
    sync(ms[i]);
  }
  return 0;
  API_CATCH(osh::last_error())
}

int osh_b200_adapt_concurrent(osh_t* meshes, unsigned n, double sf, double gq, unsigned nl,
    unsigned mo, unsigned nthreads, unsigned long long budget_bytes, unsigned* changed,
    int* status)
{
  API_TRY
  need(meshes != nullptr || n == 0, "meshes is NULL");
  std::vector<Mesh*> ms(n);
  for (unsigned i = 0; i < n; ++i) {
    need(meshes[i] != nullptr, "a mesh handle is NULL");
    ms[i] = M(meshes[i]);
    for (unsigned j = 0; j < i; ++j) need(ms[j] != ms[i], "a mesh appears twice");
  }
  t_batch_res.clear();
  osh::AdaptParams ap{sf, gq, nl, mo};
  osh::adapt_concurrent(ms, ap, nthreads, budget_bytes, t_batch_res);
  for (unsigned i = 0; i < n; ++i) {
    if (changed) changed[i] = t_batch_res[i].changed;
    if (status) status[i] = t_batch_res[i].status;
    sync(ms[i]);
  }
  return 0;
  API_CATCH(osh::last_error())
}

#define SV(h) reinterpret_cast<osh::Server*>(h)

osh_b200_server_t osh_b200_server_new(double sf, double gq, unsigned nl, unsigned mo,
    unsigned long long budget)
{
  API_TRY
  osh::AdaptParams ap{sf, gq, nl, mo};
  return reinterpret_cast<osh_b200_server_t>(osh::server_new(ap, budget));
  API_CATCH(nullptr)
}

void osh_b200_server_free(osh_b200_server_t sv)
{
  API_TRY
  osh::server_free(SV(sv));
  API_CATCH_VOID
}

int osh_b200_server_submit(osh_b200_server_t sv, unsigned dim, unsigned nverts,
    double const* coords, unsigned nelems, unsigned const* conn, double const* size)
{
  API_TRY
  need(sv != nullptr, "server is NULL");
  return (int)osh::server_submit(SV(sv), dim, nverts, coords, nelems, conn, size);
  API_CATCH(-1)
}

void osh_b200_server_set_union_elems(osh_b200_server_t sv, unsigned long long n)
{
  API_TRY
  need(sv != nullptr, "server is NULL");
  osh::server_set_union_elems(SV(sv), n);
  API_CATCH_VOID
}

int osh_b200_server_step(osh_b200_server_t sv)
{
  API_TRY
  need(sv != nullptr, "server is NULL");
  return (int)osh::server_step(SV(sv));
  API_CATCH(-1)
}

void osh_b200_server_start(osh_b200_server_t sv)
{
  API_TRY
  need(sv != nullptr, "server is NULL");
  osh::server_start(SV(sv));
  API_CATCH_VOID
}

void osh_b200_server_stop(osh_b200_server_t sv)
{
  API_TRY
  need(sv != nullptr, "server is NULL");
  osh::server_stop(SV(sv));
  API_CATCH_VOID
}

int osh_b200_server_wait(osh_b200_server_t sv, double timeout_s)
{
  API_TRY
  need(sv != nullptr, "server is NULL");
  return osh::server_wait(SV(sv), timeout_s);
  API_CATCH(-1)
}

unsigned osh_b200_server_poll(osh_b200_server_t sv, unsigned* ids, unsigned max_ids)
{
  API_TRY
  need(sv != nullptr, "server is NULL");
  std::vector<u32> r = osh::server_poll(SV(sv), ids ? max_ids : 0);
  for (size_t i = 0; i < r.size(); ++i) ids[i] = r[i];
  return (unsigned)r.size();
  API_CATCH(0)
}

osh_t osh_b200_server_take(osh_b200_server_t sv, unsigned id)
{
  API_TRY
  need(sv != nullptr, "server is NULL");
  return reinterpret_cast<osh_t>(osh::server_take(SV(sv), id));
  API_CATCH(nullptr)
}

int osh_b200_server_job_info(osh_b200_server_t sv, unsigned id, double* t_submit,
    double* t_admit, double* t_done, unsigned* passes, double* elems_in, int* status)
{
  API_TRY
  need(sv != nullptr, "server is NULL");
  osh::ServeJobInfo r = osh::server_job_info(SV(sv), id);
  if (t_submit) *t_submit = r.t_submit;
  if (t_admit) *t_admit = r.t_admit;
  if (t_done) *t_done = r.t_done;
  if (passes) *passes = r.passes;
  if (elems_in) *elems_in = r.elems_in;
  if (status) *status = r.status;
  return r.finished ? 1 : 0;
  API_CATCH(-1)
}

void osh_b200_server_stats(osh_b200_server_t sv, unsigned* steps, unsigned* active,
    unsigned* queued, unsigned long long* reserved, double* now)
{
  API_TRY
  need(sv != nullptr, "server is NULL");
  osh::ServeStats r = osh::server_stats(SV(sv));
  if (steps) *steps = r.steps;
  if (active) *active = r.active;
  if (queued) *queued = r.queued;
  if (reserved) *reserved = r.reserved;
  if (now) *now = r.now;
  API_CATCH_VOID
}

void osh_b200_server_times(osh_b200_server_t sv, double* admit, double* join,
    double* passes, double* retire)
{
  API_TRY
  need(sv != nullptr, "server is NULL");
  osh::ServeStats r = osh::server_stats(SV(sv));
  if (admit) *admit = r.secs_admit;
  if (join) *join = r.secs_join;
  if (passes) *passes = r.secs_passes;
  if (retire) *retire = r.secs_retire;
  API_CATCH_VOID
}

void osh_b200_element_gradients(osh_t h, char const* name)
{
  API_TRY
  need(h && name, "mesh or name is NULL");
  osh::element_gradients(*M(h), name);
  sync(M(h));
  API_CATCH_VOID
}

void osh_b200_recover_by_volume(osh_t h, char const* name)
{
  API_TRY
  need(h && name, "mesh or name is NULL");
  osh::recover_by_volume(*M(h), name);
  sync(M(h));
  API_CATCH_VOID
}

void osh_b200_size_from_hessian(osh_t h, char const* hess_name, double const* weights,
    double min_h, double max_h)
{
  API_TRY
  need(h && hess_name, "mesh or name is NULL");
  osh::size_from_hessian(*M(h), hess_name, weights, min_h, max_h);
  sync(M(h));
  API_CATCH_VOID
}

unsigned osh_b200_warp_to_limit(osh_t h, double qual_floor)
{
  API_TRY
  need(h != nullptr, "mesh is NULL");
  u32 r = osh::warp_to_limit(*M(h), qual_floor);
  sync(M(h));
  return r;
  API_CATCH(0)
}

void osh_b200_set_fp32_filter(osh_t h, int on)
{
  API_TRY
  need(h != nullptr, "mesh is NULL");
  M(h)->fp32_filter = on != 0;
  API_CATCH_VOID
}

void osh_b200_fp32_stats(unsigned long long* decided, unsigned long long* rechecked,
    double* max_error, unsigned* bound_exceeded)
{
  API_TRY
  osh::fp32_stats_read(decided, rechecked, max_error, bound_exceeded);
  API_CATCH_VOID
}

void osh_b200_fp32_stats_reset(void)
{
  API_TRY
  osh::fp32_stats_reset();
  API_CATCH_VOID
}

void osh_b200_set_fp32_audit(int on)
{
  API_TRY
  osh::fp32_set_audit(on != 0);
  API_CATCH_VOID
}

void osh_b200_fp32_audit_stats(unsigned long long* audited, unsigned long long* flips,
    unsigned long long* checked)
{
  API_TRY
  osh::fp32_audit_read(audited, flips, checked);
  API_CATCH_VOID
}

void osh_b200_fp32_probe_tets(unsigned n, double const* host_x, float* host_est,
    float* host_err, double* host_q64)
{
  API_TRY
  need(n == 0 || (host_x && host_est && host_err && host_q64), "null array");
  osh::fp32_probe_tets(n, host_x, host_est, host_err, host_q64);
  API_CATCH_VOID
}

void osh_b200_fp32_probe_edges(unsigned n, double const* host_x, double const* host_h,
    double thr, int* host_side, double* host_ratio64)
{
  API_TRY
  need(n == 0 || (host_x && host_h && host_side && host_ratio64), "null array");
  osh::fp32_probe_edges(n, host_x, host_h, thr, host_side, host_ratio64);
  API_CATCH_VOID
}

void osh_b200_pool_reserve(unsigned long long bytes)
{
  API_TRY
  osh::pool_reserve(bytes);
  API_CATCH_VOID
}

void osh_b200_pool_stats(unsigned long long* reserved, unsigned long long* used,
    unsigned long long* used_high, int reset_high)
{
  API_TRY
  osh::pool_stats(reserved, used, used_high, reset_high);
  API_CATCH_VOID
}

void osh_b200_write_vtk_opts(osh_t h, char const* filename, int ascii, int compress)
{
  API_TRY
  need(h != nullptr && filename != nullptr, "mesh or filename is NULL");
  osh::write_vtk(*M(h), filename, ascii != 0, compress != 0);
  API_CATCH_VOID
}

unsigned osh_b200_has_dim(osh_t h, unsigned dim)
{
  API_TRY
  need(h != nullptr, "mesh is NULL");
  Mesh* m = M(h);
  return dim <= m->dim && m->has_dim(dim) ? 1u : 0u;
  API_CATCH(0)
}

unsigned long long osh_b200_digest(osh_t h)
{
  API_TRY
  return osh::mesh_digest(*M(h));
  API_CATCH(0)
}

void osh_b200_batch_stats(unsigned* unions, unsigned* steps, unsigned* union_passes,
    unsigned* mesh_passes, double* elems_in)
{
  osh::BatchStats const& b = osh::last_batch_stats();
  if (unions) *unions = b.unions;
  if (steps) *steps = b.steps;
  if (union_passes) *union_passes = b.union_passes;
  if (mesh_passes) *mesh_passes = b.mesh_passes;
  if (elems_in) *elems_in = b.elems_in;
}

void osh_b200_batch_times(double* concat, double* passes, double* split)
{
  osh::BatchStats const& b = osh::last_batch_stats();
  if (concat) *concat = b.secs_concat;
  if (passes) *passes = b.secs_passes;
  if (split) *split = b.secs_split;
}

void osh_b200_batch_mesh_stats(unsigned i, unsigned* passes, double* elems_in)
{
  bool ok = i < t_batch_res.size();
  if (passes) *passes = ok ? t_batch_res[i].passes : 0;
  if (elems_in) *elems_in = ok ? t_batch_res[i].elems_in : 0;
}

double osh_b200_min_quality(osh_t h)
{
  API_TRY
  return M(h)->min_quality();
  API_CATCH(DBL_MAX)
}

void osh_b200_last_pass(unsigned* op, unsigned* ein, unsigned* eout, unsigned* nsel,
    unsigned* rounds)
{
  osh::PassStats const& st = osh::last_pass_stats();
  if (op) *op = st.op;
  if (ein) *ein = st.elems_in;
  if (eout) *eout = st.elems_out;
  if (nsel) *nsel = st.nselected;
  if (rounds) *rounds = st.indset_rounds;
}


unsigned osh_b200_refine_sets(osh_t h, double qf, unsigned* cand, unsigned* good,
    double* quals, unsigned* ind)
{
  API_TRY
  Mesh* m = M(h);
  u32 ne = m->count(1);
  DevOut<u32> a(cand, ne, m->s), b(good, ne, m->s), d(ind, ne, m->s);
  DevOut<double> c(quals, ne, m->s);
  u32 r = osh::refine_sets(*m, qf, a.d, b.d, c.d, d.d);
  a.back();
  b.back();
  c.back();
  d.back();
  sync(m);
  return r;
  API_CATCH(0)
}

unsigned osh_b200_coarsen_sets(osh_t h, double qf, double sf, unsigned* cs, unsigned* cc,
    unsigned* cq, double* q2, unsigned* cand, double* colq, unsigned* ind, unsigned* gv)
{
  API_TRY
  Mesh* m = M(h);
  u32 ne = m->count(1), nv = m->count(0);
  DevOut<u32> a(cs, ne, m->s), b(cc, ne, m->s), c(cq, ne, m->s), e(cand, nv, m->s),
      g(ind, nv, m->s), k(gv, nv, m->s);
  DevOut<double> d(q2, (size_t)ne * 2, m->s), f(colq, nv, m->s);
  u32 r = osh::coarsen_sets(*m, qf, sf, a.d, b.d, c.d, d.d, e.d, f.d, g.d, k.d);
  a.back();
  b.back();
  c.back();
  d.back();
  e.back();
  f.back();
  g.back();
  k.back();
  sync(m);
  return r;
  API_CATCH(0)
}

unsigned osh_b200_swap_sets(osh_t h, double gq, unsigned nl, unsigned* sl, unsigned* cand,
    unsigned* inter, unsigned* good, double* quals, unsigned* rs, unsigned* ind)
{
  API_TRY
  Mesh* m = M(h);
  need(m->dim == 3, "swap needs a 3D mesh");
  u32 ne = m->count(1), nel = m->count(3);
  DevOut<u32> a(sl, nel, m->s), b(cand, ne, m->s), c(inter, ne, m->s), d(good, ne, m->s),
      f(rs, ne, m->s), g(ind, ne, m->s);
  DevOut<double> e(quals, ne, m->s);
  u32 r = osh::swap_sets(*m, gq, nl, a.d, b.d, c.d, d.d, e.d, f.d, g.d);
  a.back();
  b.back();
  c.back();
  d.back();
  e.back();
  f.back();
  g.back();
  sync(m);
  return r;
  API_CATCH(0)
}

osh_t osh_b200_new_reduced(unsigned dim, unsigned nverts, double const* coords,
    unsigned nelems, unsigned const* conn)
{
  API_TRY
  need(dim >= 2 && dim <= 3, "elem_dim must be 2 or 3");
  Mesh* m = new Mesh(dim, false, false, nullptr);
  try {
    m->set_ents(0, nverts, nullptr);
    u32 vpe = osh::deg(dim, 0);
    u32* c = osh::dalloc<u32>((size_t)nelems * vpe, m->s);
    CK(cudaMemcpyAsync(c, conn, sizeof(u32) * nelems * vpe, cudaMemcpyHostToDevice, m->s));
    m->set_ents(dim, nelems, c);
    double* x = osh::dalloc<double>((size_t)nverts * 3, m->s);
    CK(cudaMemcpyAsync(x, coords, sizeof(double) * nverts * 3, cudaMemcpyHostToDevice, m->s));
    m->add_tag(0, osh::T_F64, "coordinates", 3, osh::X_NOT, x);
    sync(m);
  } catch (...) {
    delete m;
    throw;
  }
  return reinterpret_cast<osh_t>(m);
  API_CATCH(nullptr)
}

void osh_b200_derive_model(osh_t h, double crease)
{
  API_TRY
  M(h)->derive_model(crease);
  sync(M(h));
  API_CATCH_VOID
}

osh_t osh_b200_clone(osh_t h)
{
  API_TRY
  return reinterpret_cast<osh_t>(M(h)->clone());
  API_CATCH(nullptr)
}

void osh_b200_make_parallel(osh_t h)
{
  API_TRY
  M(h)->make_parallel();
  sync(M(h));
  API_CATCH_VOID
}

static u64 splitmix64(u64* s)
{
  u64 z = (*s += 0x9E3779B97F4A7C15ul);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ul;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBul;
  return z ^ (z >> 31);
}

static double unit_draw(u64* s)
{
  return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
}

void osh_b200_box(unsigned n, unsigned long seed, double pert, double* coords,
    unsigned* conn, double* center)
{
  // the single-cube split of tables.cpp:29-36 and its corner coordinates
  static u32 const split[6][4] = {{0, 1, 2, 6}, {2, 3, 0, 6}, {0, 3, 7, 6},
      {7, 4, 0, 6}, {0, 4, 5, 6}, {5, 1, 0, 6}};
  static u32 const corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
      {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  u32 n1 = n + 1;
  u64 s = seed;
  double amp = pert / (double)n;
  for (u32 k = 0; k < n1; ++k)
    for (u32 j = 0; j < n1; ++j)
      for (u32 i = 0; i < n1; ++i) {
        size_t v = ((size_t)k * n1 + j) * n1 + i;
        double* x = coords + v * 3;
        x[0] = (double)i / (double)n;
        x[1] = (double)j / (double)n;
        x[2] = (double)k / (double)n;
        if (i > 0 && i < n && j > 0 && j < n && k > 0 && k < n)
          for (u32 c = 0; c < 3; ++c) x[c] = x[c] + amp * (2.0 * unit_draw(&s) - 1.0);
      }
  if (center)
    for (u32 c = 0; c < 3; ++c) center[c] = 0.3 + 0.4 * unit_draw(&s);
  for (u32 k = 0; k < n; ++k)
    for (u32 j = 0; j < n; ++j)
      for (u32 i = 0; i < n; ++i) {
        size_t hx = ((size_t)k * n + j) * n + i;
        for (u32 t = 0; t < 6; ++t)
          for (u32 c = 0; c < 4; ++c) {
            u32 const* cc = corner[split[t][c]];
            conn[(hx * 6 + t) * 4 + c] = ((k + cc[2]) * n1 + (j + cc[1])) * n1 + (i + cc[0]);
          }
      }
}

void osh_b200_add_tag(osh_t h, unsigned dim, char const* name, unsigned type,
    unsigned ncomps, unsigned transfer, void const* host)
{
  API_TRY
  Mesh* m = M(h);
  need(dim <= m->dim && type <= 3 && name, "bad tag");
  size_t bytes = (size_t)m->count(dim) * ncomps * osh::tag_esz(type);
  void* d = osh::dev_alloc(bytes, m->s);
  if (bytes) CK(cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, m->s));
  m->add_tag(dim, type, name, ncomps, transfer, d);
  sync(m);
  API_CATCH_VOID
}

unsigned osh_b200_ntags(osh_t h, unsigned dim)
{
  return dim <= M(h)->dim ? (unsigned)M(h)->tags[dim].size() : 0u;
}

char const* osh_b200_tag_name(osh_t h, unsigned dim, unsigned i)
{
  API_TRY
  return tag_at(M(h), dim, i)->name.c_str();
  API_CATCH(nullptr)
}

void osh_b200_tag_info(osh_t h, unsigned dim, unsigned i, unsigned* type, unsigned* ncomps,
    unsigned* transfer)
{
  API_TRY
  osh::Tag* t = tag_at(M(h), dim, i);
  if (type) *type = t->type;
  if (ncomps) *ncomps = t->ncomps;
  if (transfer) *transfer = t->transfer;
  API_CATCH_VOID
}

void const* osh_b200_tag_data(osh_t h, unsigned dim, unsigned i)
{
  API_TRY
  return tag_at(M(h), dim, i)->data;
  API_CATCH(nullptr)
}

void osh_b200_set_globals(osh_t h, unsigned dim, unsigned long const* host)
{
  API_TRY
  Mesh* m = M(h);
  need(dim <= m->dim, "bad dimension");
  u32 n = m->count(dim);
  u64* g = osh::dalloc<u64>(n, m->s);
  CK(cudaMemcpyAsync(g, host, sizeof(u64) * n, cudaMemcpyHostToDevice, m->s));
  m->set_globals(dim, g);
  m->parallel = true;
  sync(m);
  API_CATCH_VOID
}

unsigned const* osh_b200_dual(osh_t h)
{
  API_TRY
  u32 const* r = M(h)->ask_dual();
  sync(M(h));
  return r;
  API_CATCH(nullptr)
}

void osh_b200_qualities(osh_t h, double* out)
{
  API_TRY
  Mesh* m = M(h);
  double const* q = m->qualities();
  CK(cudaMemcpyAsync(out, q, sizeof(double) * m->count(m->dim), cudaMemcpyDeviceToHost, m->s));
  sync(m);
  API_CATCH_VOID
}

void osh_b200_edge_lengths(osh_t h, double* out)
{
  API_TRY
  Mesh* m = M(h);
  double* l = m->measure_edges();
  CK(cudaMemcpyAsync(out, l, sizeof(double) * m->count(1), cudaMemcpyDeviceToHost, m->s));
  osh::dev_free(l, m->s);
  sync(m);
  API_CATCH_VOID
}

void osh_b200_copy_to_host(void* dst, void const* src, size_t bytes)
{
  API_TRY
  CK(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
  API_CATCH_VOID
}

void osh_b200_copy_to_device(void* dst, void const* src, size_t bytes)
{
  API_TRY
  CK(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
  API_CATCH_VOID
}

void osh_b200_copy_to_host_async(osh_t h, void* dst, void const* src, size_t bytes)
{
  API_TRY
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, M(h)->s));
  API_CATCH_VOID
}

void osh_b200_copy_to_device_async(osh_t h, void* dst, void const* src, size_t bytes)
{
  API_TRY
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, M(h)->s));
  API_CATCH_VOID
}

void osh_b200_synchronize(osh_t h)
{
  API_TRY
  sync(M(h));
  API_CATCH_VOID
}

void osh_b200_adapt_stats(unsigned* passes, double* elems_in)
{
  osh::AdaptStats const& st = osh::last_adapt_stats();
  if (passes) *passes = st.passes;
  if (elems_in) *elems_in = st.elems_in;
}

unsigned long long osh_b200_launch_count(void) { return osh::launch_count(); }
unsigned long long osh_b200_sync_count(void) { return osh::sync_count(); }
void osh_b200_host_stats(unsigned long long* allocs, double* sync_wait_seconds)
{
  osh::host_stats(allocs, sync_wait_seconds);
}

unsigned osh_b200_tuning_count(void) { return osh::TK_NKEYS; }
char const* osh_b200_tuning_name(unsigned i) { return osh::tune_name(i); }
int osh_b200_tuning_get(char const* name, unsigned* value) { return osh::tune_get(name, value); }
int osh_b200_tuning_set(char const* name, unsigned value) { return osh::tune_set(name, value); }
int osh_b200_tuning_load(char const* path) { return osh::tune_load(path); }

int osh_b200_selftest_scan_wait(unsigned spin_limit)
{
  API_TRY
  return osh::selftest_scan_wait(spin_limit);
  API_CATCH(osh::last_error())
}

int osh_b200_exscan_u32(unsigned const* in, unsigned* out, unsigned n, void* stream, int check)
{
  API_TRY
  need(out != nullptr && (in != nullptr || n == 0), "exscan: null array");
  uintptr_t const a = reinterpret_cast<uintptr_t>(in), b = reinterpret_cast<uintptr_t>(out);
  need(n == 0 || b + 4ull * ((u64)n + 1) <= a || a + 4ull * n <= b, "exscan: in and out overlap");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  osh::exscan_u32(in, out, n, s, nullptr, nullptr);
  if (check) osh::check_device_timeouts(s);
  return 0;
  API_CATCH(osh::last_error())
}

void osh_b200_set_stream(osh_t h, void* stream)
{
  API_TRY
  M(h)->use_stream(static_cast<cudaStream_t>(stream));
  API_CATCH_VOID
}

void osh_b200_release_stream(void* stream)
{
  API_TRY
  osh::release_stream_scratch(static_cast<cudaStream_t>(stream));
  API_CATCH_VOID
}

void osh_b200_probe_enable(unsigned mask) { osh::probe_enable(mask); }

void osh_b200_probe_reset(void)
{
  API_TRY
  osh::probe_reset();
  API_CATCH_VOID
}

unsigned osh_b200_probe_count(void) { return osh::P_NPROBES; }
char const* osh_b200_probe_name(unsigned id) { return osh::probe_name(id); }

void osh_b200_probe_read(unsigned id, unsigned* launches, double* ms, double* bytes)
{
  API_TRY
  need(id < osh::P_NPROBES, "bad probe id");
  osh::probe_read(id, launches, ms, bytes);
  API_CATCH_VOID
}

unsigned osh_b200_swap_table(unsigned rs, unsigned* ntri, unsigned* nmesh, unsigned* nint,
    unsigned* tris, unsigned* iedges)
{
  if (rs < 3 || rs > osh::MAX_EDGE_SWAP) return 0;
  osh::swap_table_host(rs, ntri, nmesh, nint, tris, iedges);
  return 1;
}

}  // extern "C"
