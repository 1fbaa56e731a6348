// The single-precision filter's estimates evaluated for caller-given
// elements and edges, beside the double values the passes compute: the
// device side of the filter's error-bound tests (the same device functions
// the refine, coarsen and swap kernels call).
#include "runtime.hpp"

namespace osh {

__global__ void k_probe_tets(u32 n, double const* __restrict__ x, float* __restrict__ est,
    float* __restrict__ err, double* __restrict__ q64)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double ex[4][3];
  for (u32 v = 0; v < 4; ++v)
    for (u32 c = 0; c < 3; ++c) ex[v][c] = x[(size_t)i * 12 + v * 3 + c];
  Q32 q = tet_quality_f32(ex, tet_k6_f32());
  est[i] = q.q;
  err[i] = q.err;
  q64[i] = tet_quality(ex, perfect_tet_quality());
}

__global__ void k_probe_edges(u32 n, double const* __restrict__ x, double const* __restrict__ h,
    double thr, int* __restrict__ side, double* __restrict__ ratio64)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double xa[3], xb[3];
  for (u32 c = 0; c < 3; ++c) {
    xa[c] = x[(size_t)i * 6 + c];
    xb[c] = x[(size_t)i * 6 + 3 + c];
  }
  side[i] = edge_ratio_side_f32(xa, xb, h[i * 2], h[i * 2 + 1], thr);
  double len = sqrt(sqdist3(xb, xa));
  double want = (h[i * 2] + h[i * 2 + 1]) / 2;
  ratio64[i] = len / want;
}

namespace {
template <class T>
T* upload(T const* host, size_t n, cudaStream_t s)
{
  T* d = dalloc<T>(n ? n : 1, s);
  if (n) CK(cudaMemcpyAsync(d, host, n * sizeof(T), cudaMemcpyHostToDevice, s));
  return d;
}
template <class T>
void download(T* host, T const* d, size_t n, cudaStream_t s)
{
  if (n) CK(cudaMemcpyAsync(host, d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
}
}  // namespace

void fp32_probe_tets(u32 n, double const* host_x, float* est, float* err, double* q64)
{
  cudaStream_t s = 0;
  double* x = upload(host_x, (size_t)n * 12, s);
  float* e = dalloc<float>(2 * (size_t)n + 2, s);
  double* q = dalloc<double>((size_t)n + 1, s);
  if (n) {
    CK(launch_kernel(k_probe_tets, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, x, e, e + n, q));
    CK_LAUNCH();
  }
  download(est, e, n, s);
  download(err, e + n, n, s);
  download(q64, q, n, s);
  stream_sync(s);
  dev_free(x, s);
  dev_free(e, s);
  dev_free(q, s);
}

void fp32_probe_edges(u32 n, double const* host_x, double const* host_h, double thr,
    int* side, double* ratio64)
{
  cudaStream_t s = 0;
  double* x = upload(host_x, (size_t)n * 6, s);
  double* h = upload(host_h, (size_t)n * 2, s);
  int* sd = dalloc<int>((size_t)n + 1, s);
  double* r = dalloc<double>((size_t)n + 1, s);
  if (n) {
    CK(launch_kernel(k_probe_edges, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, x, h, thr, sd, r));
    CK_LAUNCH();
  }
  download(side, sd, n, s);
  download(ratio64, r, n, s);
  stream_sync(s);
  dev_free(x, s);
  dev_free(h, s);
  dev_free(sd, s);
  dev_free(r, s);
}

}  // namespace osh
