// Size-field producers on the device: element gradients of vertex fields
// (element_gradients.cpp:15-91 with jacobian.cpp:7-66), recovery of element
// fields to vertices weighted by element volume (recover_by_volume.cpp:10-68),
// an isotropic size from recovered Hessians (size_from_hessian.cpp:12-72), and
// warping coordinates as far as a quality floor allows
// (warp_to_limit.cpp:14-81). Every arithmetic step follows the reference's
// order, so results are bit-identical to its CPU build.
#include <cfloat>
#include <string>

#include "fields.hpp"

namespace osh {

namespace {

// algebra.hpp's helpers, in their operation order
__device__ inline void cross_ref(double const* a, double const* b, double* c)
{
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ inline double dot_ref(double const* a, double const* b, u32 n)
{
  double d = 0;
  for (u32 i = 0; i < n; ++i) d += a[i] * b[i];
  return d;
}

// invert_jacobian (jacobian.cpp:20-61) for 1-, 2- and 3-simplices
__device__ void invert_jacobian(u32 dim, double in[3][3], double out[3][3])
{
  if (dim == 3) {
    // invert_3x3 (algebra.hpp): cofactor rows scaled by 1/det, transposed
    double tmp[3][3], c[3];
    cross_ref(in[0], in[1], c);
    double d = dot_ref(in[2], c, 3);
    cross_ref(in[1], in[2], tmp[0]);
    cross_ref(in[2], in[0], tmp[1]);
    cross_ref(in[0], in[1], tmp[2]);
    double s = 1.0 / d;
    for (u32 i = 0; i < 3; ++i)
      for (u32 j = 0; j < 3; ++j) tmp[i][j] = tmp[i][j] * s;
    for (u32 i = 0; i < 3; ++i)
      for (u32 j = 0; j < 3; ++j) out[i][j] = tmp[j][i];
  } else if (dim == 2) {
    double nrm[2][2];
    for (u32 i = 0; i < 2; ++i)
      for (u32 j = 0; j < 2; ++j) {
        nrm[i][j] = 0;
        for (u32 k = 0; k < 3; ++k) nrm[i][j] += in[i][k] * in[j][k];
      }
    double d = nrm[0][0] * nrm[1][1] - nrm[0][1] * nrm[1][0];
    double inv[2][2] = {{nrm[1][1] / d, -nrm[0][1] / d}, {-nrm[1][0] / d, nrm[0][0] / d}};
    for (u32 i = 0; i < 3; ++i)
      for (u32 j = 0; j < 3; ++j) out[i][j] = 0;
    for (u32 i = 0; i < 3; ++i)
      for (u32 j = 0; j < 2; ++j)
        for (u32 k = 0; k < 2; ++k) out[i][j] += in[k][i] * inv[k][j];
  } else {
    double msq = dot_ref(in[0], in[0], 3);
    for (u32 i = 0; i < 3; ++i) out[i][0] = in[0][i] / msq;
    for (u32 i = 0; i < 3; ++i)
      for (u32 j = 1; j < 3; ++j) out[i][j] = 0;
  }
}

__global__ void k_element_gradients(u32 dim, u32 ne, u32 const* __restrict__ voe,
    double const* __restrict__ x, u32 nc, double const* __restrict__ f,
    double* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  u32 vpe = dim + 1;
  u32 const* ve = voe + (size_t)i * vpe;
  double ex[4][3];
  for (u32 j = 0; j < vpe; ++j) load3(x, ve[j], ex[j]);
  // element_jacobian: column j is x[j+1] - x[0]
  double jac[3][3];
  for (u32 a = 0; a < 3; ++a)
    for (u32 b = 0; b < 3; ++b) jac[a][b] = 0;
  for (u32 a = 0; a < dim; ++a)
    for (u32 b = 0; b < 3; ++b) jac[b][a] = ex[a + 1][b] - ex[0][b];
  double jaci[3][3];
  invert_jacobian(dim, jac, jaci);
  double* g = out + (size_t)i * nc * 3;
  for (u32 k = 0; k < nc * 3; ++k) g[k] = 0;
  for (u32 j = 0; j < dim; ++j)
    for (u32 k = 0; k < nc; ++k)
      for (u32 l = 0; l < 3; ++l)
        g[k * 3 + l] += jaci[j][l] * (f[(size_t)ve[j + 1] * nc + k] - f[(size_t)ve[0] * nc + k]);
}

__global__ void k_recover_by_volume(u32 nv, u32 const* __restrict__ offs,
    u32 const* __restrict__ adj, double const* __restrict__ sizes, u32 nc,
    double const* __restrict__ f, double* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  double* o = out + (size_t)i * nc;
  for (u32 k = 0; k < nc; ++k) o[k] = 0;
  double size_sum = 0;
  for (u32 j = offs[i]; j < offs[i + 1]; ++j) {
    u32 e = adj[j];
    double es = sizes[e];
    size_sum += es;
    for (u32 k = 0; k < nc; ++k) o[k] += es * f[(size_t)e * nc + k];
  }
  for (u32 k = 0; k < nc; ++k) o[k] /= size_sum;
}

__global__ void k_size_from_hessian(u32 nv, u32 nhc, double const* __restrict__ hess,
    double const* __restrict__ w, u32 nsol, double min_h, double max_h,
    double* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  double const* hs = hess + (size_t)i * nhc;
  double total = 0;
  for (u32 j = 0; j < nsol; ++j) {
    double norm = sqrt(dot_ref(hs, hs, 9));
    double hw = w ? w[j] : 1.0;
    total += hw * norm;
    hs += 9;
  }
  // clamp (size_from_hessian.cpp:34-40)
  double o = max_h - total;
  if (o < min_h) o = min_h;
  out[i] = o;
}

__global__ void k_axpy(u32 n, double a, double const* __restrict__ x,
    double const* __restrict__ y, double* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a * x[i] + y[i];
}

__global__ void k_min_quality(u32 dim, u32 ne, u32 const* __restrict__ voe,
    double const* __restrict__ x, unsigned long long* minkey)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long key = ~0ull;
  if (i < ne) {
    u32 vpe = dim + 1;
    double ex[4][3];
    for (u32 j = 0; j < vpe; ++j) load3(x, voe[(size_t)i * vpe + j], ex[j]);
    double q = elem_quality(dim, ex, 1);
    key = order_key(q);
  }
  for (int o = 16; o; o >>= 1) {
    unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
    key = other < key ? other : key;
  }
  if ((threadIdx.x & 31) == 0 && key != ~0ull) atomicMin(minkey, key);
}

}  // namespace

void element_gradients(Mesh& m, char const* name)
{
  cudaStream_t s = m.s;
  Tag* t = m.find_tag(0, name);
  if (!t || t->type != T_F64) throw Failure(E_ARG, std::string("no vertex field ") + name);
  u32 dim = m.dim, ne = m.count(dim), nc = t->ncomps;
  double* out = dalloc<double>((size_t)ne * nc * 3, s);
  if (ne) {
    CK(launch_kernel(k_element_gradients, dim3(grid_for(ne)), dim3(BLOCK), 0, s, dim, ne, m.ask_down(dim, 0), m.coords(),
        nc, static_cast<double const*>(t->data), out));
    CK_LAUNCH();
  }
  m.add_tag(dim, T_F64, (std::string("grad_") + name).c_str(), nc * 3, X_NOT, out);
}

void recover_by_volume(Mesh& m, char const* name)
{
  cudaStream_t s = m.s;
  u32 dim = m.dim;
  Tag* t = m.find_tag(dim, name);
  if (!t || t->type != T_F64) throw Failure(E_ARG, std::string("no element field ") + name);
  u32 nv = m.count(0), nc = t->ncomps;
  UpAdj const& ve = m.ask_up(0, dim, true);
  double* sizes = m.element_sizes();
  double* out = dalloc<double>((size_t)nv * nc, s);
  if (nv) {
    CK(launch_kernel(k_recover_by_volume, dim3(grid_for(nv)), dim3(BLOCK), 0, s, nv, ve.offs, ve.adj, sizes, nc,
        static_cast<double const*>(m.find_tag(dim, name)->data), out));
    CK_LAUNCH();
  }
  dev_free(sizes, s);
  m.add_tag(0, T_F64, name, nc, X_NOT, out);
}

void size_from_hessian(Mesh& m, char const* hess_name, double const* weights, double min_h,
    double max_h)
{
  cudaStream_t s = m.s;
  Tag* t = m.find_tag(0, hess_name);
  if (!t || t->type != T_F64) throw Failure(E_ARG, std::string("no vertex field ") + hess_name);
  if (t->ncomps % 9 || !(max_h > min_h) || !(min_h > 0))
    throw Failure(E_ARG, "size_from_hessian needs 9k components and 0 < min_h < max_h");
  u32 nv = m.count(0), nsol = t->ncomps / 9;
  double* w = nullptr;
  if (weights) {
    for (u32 j = 0; j < nsol; ++j)
      if (!(weights[j] >= 0)) throw Failure(E_ARG, "negative Hessian weight");
    w = dalloc<double>(nsol, s);
    CK(cudaMemcpyAsync(w, weights, sizeof(double) * nsol, cudaMemcpyHostToDevice, s));
  }
  double* out = dalloc<double>(nv, s);
  if (nv) {
    CK(launch_kernel(k_size_from_hessian, dim3(grid_for(nv)), dim3(BLOCK), 0, s, nv, t->ncomps,
        static_cast<double const*>(t->data), w, nsol, min_h, max_h, out));
    CK_LAUNCH();
  }
  stream_sync(s);
  dev_free(w, s);
  m.add_tag(0, T_F64, "adapt_size", 1, X_NOT, out);
}

static double min_quality_of(Mesh& m, double const* x)
{
  cudaStream_t s = m.s;
  u32 ne = m.count(m.dim);
  unsigned long long* mk = reinterpret_cast<unsigned long long*>(m.mb->dev + 30);
  CK(cudaMemsetAsync(mk, 0xff, sizeof(unsigned long long), s));
  if (ne) {
    CK(launch_kernel(k_min_quality, dim3(grid_for(ne)), dim3(BLOCK), 0, s, m.dim, ne, m.ask_down(m.dim, 0), x, mk));
    CK_LAUNCH();
  }
  m.mb->fetch(s, 32);
  unsigned long long k;
  std::memcpy(&k, m.mb->host + 30, sizeof(k));
  return k == ~0ull ? DBL_MAX : from_order_key(k);
}

u32 warp_to_limit(Mesh& m, double qual_floor)
{
  cudaStream_t s = m.s;
  Tag* xt = m.find_tag(0, "coordinates");
  Tag* wt = m.find_tag(0, "warp");
  if (!xt || !wt || wt->ncomps != 3) throw Failure(E_ARG, "warp_to_limit needs a 3-vector warp");
  u32 n = m.count(0) * 3;
  double const* x = static_cast<double const*>(xt->data);
  double const* w = static_cast<double const*>(wt->data);
  double* xo = dalloc<double>(n, s);
  double factor = 1;
  u32 hit = 0;
  auto apply = [&]() {
    if (n) {
      CK(launch_kernel(k_axpy, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, factor, w, x, xo));
      CK_LAUNCH();
    }
  };
  apply();
  // exceeds_limit (warp_to_limit.cpp:14-29); halving ends after at most
  // 64 steps, when the warp no longer moves any coordinate
  for (u32 it = 0; min_quality_of(m, xo) < qual_floor; ++it) {
    if (it >= 1100) throw Failure(E_NOCONVERGE, "warp_to_limit: quality floor not reached");
    hit = 1;
    factor /= 2;
    apply();
  }
  double* wo = dalloc<double>(n, s);
  if (n) {
    CK(launch_kernel(k_axpy, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, -factor, w, w, wo));
    CK_LAUNCH();
  }
  m.remove_tag(0, "coordinates");
  m.remove_tag(0, "warp");
  m.add_tag(0, T_F64, "coordinates", 3, X_NOT, xo);
  m.add_tag(0, T_F64, "warp", 3, X_NOT, wo);
  dev_free(m.qual_cache, s);
  m.qual_cache = nullptr;
  return hit ? 0u : 1u;
}

}  // namespace osh
