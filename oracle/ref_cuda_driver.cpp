// Test and measurement infrastructure only (never shipped, never timed as
// the product): a thin extern "C" driver over the reference built in its own
// CUDA loop mode (loop_cuda.hpp: one thread per item, cudaMalloc per array,
// Thrust for scans, reductions and sorts), compiled from the reference's own
// sources for sm_100a by oracle/Makefile. bench.py times its mesh_adapt on
// the same input as ours, so the reference's GPU path is measured beside its
// CPU path. In this mode every mesh array lives in device memory, so inputs
// and outputs cross with cudaMemcpy.
//
// Mesh set-up follows the reference's own tests (test_warp_3d.cpp:115-119).

#include <cuda_runtime.h>

#include <cstring>

#include "adapt.hpp"
#include "algebra.hpp"
#include "coarsen.hpp"
#include "derive_model.hpp"
#include "loop.hpp"
#include "mesh.hpp"
#include "parallel_mesh.hpp"
#include "quality.hpp"
#include "refine.hpp"
#include "swap.hpp"
#include "tables.hpp"
#include "tag.hpp"

using namespace omega_h;

#define M(p) reinterpret_cast<struct mesh*>(p)

namespace {
template <class T>
T* to_device(T const* host, unsigned long n)
{
  T* d = LOOP_MALLOC(T, n);
  cudaMemcpy(d, host, sizeof(T) * n, cudaMemcpyHostToDevice);
  return d;
}
}  // namespace

extern "C" {

// 0 when the CUDA runtime works here, else the cudaError_t
int refc_ready(void)
{
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) return (int)e;
  return n > 0 ? 0 : -1;
}

void* refc_new_reduced(unsigned dim, unsigned nverts, double const* coords,
    unsigned nelems, unsigned const* conn)
{
  struct mesh* m = new_mesh(dim, MESH_REDUCED, 0);
  mesh_set_ents(m, 0, nverts, 0);
  unsigned vpe = the_down_degrees[dim][0];
  mesh_set_ents(m, dim, nelems, to_device(conn, (unsigned long)nelems * vpe));
  mesh_add_tag(m, 0, TAG_F64, "coordinates", 3, to_device(coords, (unsigned long)nverts * 3));
  return m;
}

void refc_derive_model_full(void* p)
{
  mesh_derive_model(M(p), PI / 4);
  mesh_set_rep(M(p), MESH_FULL);
}

void refc_add_vertex_field(void* p, char const* name, double const* data)
{
  unsigned nv = mesh_count(M(p), 0);
  mesh_add_tag(M(p), 0, TAG_F64, name, 1, to_device(data, nv));
}

unsigned refc_adapt(void* p, double size_floor, double good_qual, unsigned nlayers,
    unsigned max_ops)
{
  unsigned r = mesh_adapt(M(p), size_floor, good_qual, nlayers, max_ops);
  cudaDeviceSynchronize();
  return r;
}

// mesh_adapt's pass sequence (adapt.cpp:47-94) with the elements entering
// each pass that changed the mesh summed, for the tets/s metric
unsigned refc_adapt_counted(void* p, double sf, double gq, unsigned nl, unsigned max_ops,
    unsigned* passes, double* elems_in)
{
  struct mesh* m = M(p);
  unsigned dim = mesh_dim(m), ops = 0;
  double in = 0;
  double qf = mesh_min_quality(m);
  if (gq < qf) qf = gq;
  unsigned before = 0;
  auto pass = [&](unsigned changed) {
    if (changed) {
      in += before;
      ++ops;
    }
    return changed != 0 && ops <= max_ops;
  };
  for (;;) {
    before = mesh_count(m, dim);
    if (!pass(refine_by_size(m, qf))) break;
  }
  for (;;) {
    before = mesh_count(m, dim);
    if (!pass(coarsen_by_size(m, qf, sf))) break;
  }
  while (mesh_min_quality(m) < gq && ops <= max_ops) {
    before = mesh_count(m, dim);
    if (dim == 3 && pass(swap_slivers(m, gq, nl))) continue;
    before = mesh_count(m, dim);
    if (pass(coarsen_slivers(m, gq, nl))) continue;
    break;
  }
  cudaDeviceSynchronize();
  *passes = ops;
  *elems_in = in;
  return ops > 0;
}

unsigned refc_count(void* p, unsigned dim) { return mesh_count(M(p), dim); }

void refc_verts_of_elems(void* p, unsigned* host_out)
{
  unsigned d = mesh_dim(M(p));
  unsigned n = mesh_count(M(p), d) * the_down_degrees[d][0];
  cudaMemcpy(host_out, mesh_ask_down(M(p), d, 0), sizeof(unsigned) * n, cudaMemcpyDeviceToHost);
}

void refc_coords(void* p, double* host_out)
{
  unsigned n = mesh_count(M(p), 0) * 3;
  cudaMemcpy(host_out, mesh_find_tag(M(p), 0, "coordinates")->d.f64, sizeof(double) * n,
      cudaMemcpyDeviceToHost);
}

// the last CUDA error of this library's runtime (0 = none)
int refc_last_error(void) { return (int)cudaGetLastError(); }

void refc_free(void* p) { free_mesh(M(p)); }

}  // extern "C"
