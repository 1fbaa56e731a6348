// Shared definitions for the sm_100a adaptation pass: entity tables, device
// geometry (quality / size) and host-side CUDA helpers.
//
// Floating point: every translation unit is compiled with -fmad=false so that
// a*b+c stays two IEEE-rounded operations, and every expression below keeps
// the operation order of the reference (algebra.hpp, size.hpp, quality.hpp).
// FP64 division and sqrt on the device are correctly rounded, as on the host,
// so per-element results are bit-identical to the reference's CPU build.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

namespace osh {

typedef unsigned u32;
typedef unsigned long u64;  // 64-bit on LP64, matches omega_h.h's globals

constexpr u32 INV = 0xffffffffu;
constexpr u32 MAX_EDGE_SWAP = 7;  // edge_swap.hpp:6
constexpr u32 MAX_PTS = 16;       // qr.hpp:6
constexpr u32 MAX_NCOMPS = 32;    // coarsen_conserve.cpp:10
constexpr u32 MAX_INDSET_ROUNDS = 100;  // indset.cpp:33

enum TagType { T_U8 = 0, T_U32 = 1, T_U64 = 2, T_F64 = 3 };
enum Transfer { X_NOT = 0, X_POINTWISE = 1, X_CONSERVE = 2, X_INHERIT = 3 };
enum Collapse { DONT_COLLAPSE = 0, COLLAPSE_BOTH = 3 };
enum IndsetState { NOT_IN_SET = 0, IN_SET = 1, UNKNOWN = 2 };

// error codes returned through osh_b200_last_error()
enum Error {
  E_OK = 0,
  E_CUDA = 1,         // a CUDA runtime call failed
  E_NOCONVERGE = 2,   // independent set did not settle in 100 rounds
  E_MAXOPS = 3,       // mesh_adapt exceeded max_passes
  E_ARG = 4,          // bad argument (dimension, missing tag, ...)
  E_NOMEM = 5,        // device allocation failed
  E_UNSUPPORTED = 6,  // entry point not available in this build
  E_TIMEOUT = 7,      // a bounded device wait gave up
  E_INVERTED = 8,     // refinement met an inverted element (reference asserts)
  E_IO = 9,           // a mesh file could not be opened, read or parsed
};

struct Failure : std::runtime_error {
  int code;
  Failure(int c, std::string const& what) : std::runtime_error(what), code(c) {}
};

void check_cuda(cudaError_t e, char const* what, char const* file, int line);
#define CK(x) ::osh::check_cuda((x), #x, __FILE__, __LINE__)
void count_launch();
#define CK_LAUNCH()                                                              \
  do {                                                                           \
    ::osh::count_launch();                                                       \
    ::osh::check_cuda(cudaGetLastError(), "kernel launch", __FILE__, __LINE__);  \
  } while (0)

inline u32 ceil_div(u64 a, u64 b) { return (u32)((a + b - 1) / b); }

// order-preserving 64-bit key of a double (min of keys = min of values)
__device__ inline unsigned long long order_key(double x)
{
  unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | (1ull << 63));
}

__host__ inline double from_order_key(unsigned long long k)
{
  unsigned long long b = (k >> 63) ? (k & ~(1ull << 63)) : ~k;
  double x;
  std::memcpy(&x, &b, sizeof(x));
  return x;
}

constexpr int BLOCK = 256;
inline u32 grid_for(u64 n) { return n ? ceil_div(n, BLOCK) : 1; }

// ---------------------------------------------------------------------------
// entity tables (tables.cpp:77-193)

__host__ __device__ constexpr u32 deg(u32 high, u32 low)
{
  return high == 0 ? (low == 0 ? 1 : 0)
       : high == 1 ? (low == 0 ? 2 : low == 1 ? 1 : 0)
       : high == 2 ? (low <= 1 ? 3 : low == 2 ? 1 : 0)
       : (low == 0 ? 4 : low == 1 ? 6 : low == 2 ? 4 : 1);
}

// local vertices of the edges of a triangle / tet, faces of a tet
__host__ __device__ inline u32 tri_edge_vert(u32 e, u32 k)
{
  return k == 0 ? e : (e + 1) % 3;  // {0,1},{1,2},{2,0}
}
__host__ __device__ inline u32 tet_edge_vert(u32 e, u32 k)
{
  // {0,1},{1,2},{2,0},{0,3},{1,3},{2,3}
  return e < 3 ? (k == 0 ? e : (e + 1) % 3) : (k == 0 ? e - 3 : 3);
}
__host__ __device__ inline u32 tet_face_vert(u32 f, u32 k)
{
  // {0,1,2},{1,0,3},{2,1,3},{0,2,3}
  constexpr u32 t = (0u << 0) | (1u << 2) | (2u << 4) | (1u << 6) | (0u << 8) |
                    (3u << 10) | (2u << 12) | (1u << 14) | (3u << 16) |
                    (0u << 18) | (2u << 20) | (3u << 22);
  return (t >> (2 * (f * 3 + k))) & 3u;
}
__host__ __device__ inline u32 tet_face_edge(u32 f, u32 k)
{
  // {0,1,2},{0,3,4},{1,4,5},{2,5,3}
  constexpr u64 t = (0ull << 0) | (1ull << 3) | (2ull << 6) | (0ull << 9) |
                    (3ull << 12) | (4ull << 15) | (1ull << 18) | (4ull << 21) |
                    (5ull << 24) | (2ull << 27) | (5ull << 30) | (3ull << 33);
  return (u32)((t >> (3 * (f * 3 + k))) & 7u);
}

// the_canonical_orders[elem][ent][sub][j][k]
__host__ __device__ inline u32 canon(u32 elem, u32 ent, u32 sub, u32 j, u32 k)
{
  if (ent == elem) return k;
  if (sub == ent) return j;
  if (ent == 1 && sub == 0) return elem == 2 ? tri_edge_vert(j, k) : tet_edge_vert(j, k);
  if (ent == 2 && sub == 0) return tet_face_vert(j, k);
  return tet_face_edge(j, k);
}

// edge opposite each tet edge {5,3,4,1,2,0}
__host__ __device__ inline u32 tet_opp_edge(u32 e)
{
  switch (e) {
    case 0: return 5;
    case 1: return 3;
    case 2: return 4;
    case 3: return 1;
    case 4: return 2;
    default: return 0;
  }
}

// the_opposite_orders[elem][dim][j]
__host__ __device__ inline u32 opp(u32 elem, u32 dim, u32 j)
{
  if (elem == 1) return 1 - j;                          // {1,0}
  if (elem == 2) return dim == 0 ? (j + 1) % 3          // {1,2,0}
                                 : (j + 2) % 3;         // {2,0,1}
  if (dim == 0) return (0x0132u >> (4 * j)) & 0xfu;     // {2,3,1,0}
  if (dim == 1) return tet_opp_edge(j);                 // {5,3,4,1,2,0}
  return (0x1023u >> (4 * j)) & 0xfu;                   // {3,2,0,1}
}

// ---------------------------------------------------------------------------
// geometry (size.hpp, quality.hpp, algebra.hpp)

struct V3 {
  double x[3];
};

__host__ __device__ inline void sub3(double const* a, double const* b, double* c)
{
  c[0] = a[0] - b[0];
  c[1] = a[1] - b[1];
  c[2] = a[2] - b[2];
}

__host__ __device__ inline void cross3(double const* a, double const* b, double* c)
{
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

__host__ __device__ inline double dot3(double const* a, double const* b)
{
  double d = 0;
  d += a[0] * b[0];
  d += a[1] * b[1];
  d += a[2] * b[2];
  return d;
}

__host__ __device__ inline double sqdist3(double const* a, double const* b)
{
  double s = 0;
  double d0 = a[0] - b[0];
  s += d0 * d0;
  double d1 = a[1] - b[1];
  s += d1 * d1;
  double d2 = a[2] - b[2];
  s += d2 * d2;
  return s;
}

// triangle_area (size.hpp:14-23)
__host__ __device__ inline double tri_area(double const* x0, double const* x1,
    double const* x2)
{
  double v0[3], v1[3], c[3];
  sub3(x1, x0, v0);
  sub3(x2, x0, v1);
  cross3(v0, v1, c);
  return sqrt(dot3(c, c)) / 2.0;
}

__host__ __device__ inline double tri_z_area(double const* x0, double const* x1,
    double const* x2)
{
  double v0[3], v1[3], c[3];
  sub3(x1, x0, v0);
  sub3(x2, x0, v1);
  cross3(v0, v1, c);
  return c[2] / 2.0;
}

// tet_volume (size.hpp:36-46)
__host__ __device__ inline double tet_volume(double const (*x)[3])
{
  double v0[3], v1[3], v2[3], c[3];
  sub3(x[1], x[0], v0);
  sub3(x[2], x[0], v1);
  sub3(x[3], x[0], v2);
  cross3(v0, v1, c);
  return dot3(c, v2) / 6.0;
}

// normalisation constants (quality.hpp:15-18), computed the same way
__host__ __device__ inline double perfect_tri_quality() { return sqrt(3.0) / 4.0; }
__host__ __device__ inline double perfect_tet_quality()
{
  double s = sqrt(perfect_tri_quality());
  return (sqrt(2.0) / 12.0) / (s * s * s);
}

// Single-precision filter for quality decisions. The estimate is formed
// from coordinates relative to the first vertex (each difference taken in
// double, then rounded), with a running bound on its error: the triple
// product and the face areas are each off by at most a few float epsilons
// of the products of the edge lengths that form them, which the bound
// scales by the same normalisation as the quality. A candidate is rejected
// on the estimate only when estimate + bound is already below the
// threshold; every other decision, and every value that is kept, comes from
// the double computation, so all decisions equal the double path's.
struct Q32 {
  float q;    // estimate of tet_quality
  float err;  // bound on |estimate - tet_quality|; inf when unbounded
};

__device__ inline float3 f3sub(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ inline float3 f3cross(float3 a, float3 b)
{
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ inline float f3dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ inline float f3norm(float3 a) { return sqrtf(f3dot(a, a)); }

__device__ inline Q32 tet_quality_f32(double const (*x)[3], float perfect)
{
  float3 d0 = make_float3((float)(x[1][0] - x[0][0]), (float)(x[1][1] - x[0][1]),
      (float)(x[1][2] - x[0][2]));
  float3 d1 = make_float3((float)(x[2][0] - x[0][0]), (float)(x[2][1] - x[0][1]),
      (float)(x[2][2] - x[0][2]));
  float3 d2 = make_float3((float)(x[3][0] - x[0][0]), (float)(x[3][1] - x[0][1]),
      (float)(x[3][2] - x[0][2]));
  float3 e12 = f3sub(d1, d0), e13 = f3sub(d2, d0), e23 = f3sub(d2, d1);
  float3 c0 = f3cross(d0, d1), c1 = f3cross(d0, e13), c2 = f3cross(e12, e23), c3 = f3cross(d1, d2);
  float sum_asq = 0.25f * (f3dot(c0, c0) + f3dot(c1, c1) + f3dot(c2, c2) + f3dot(c3, c3));
  float arms = sqrtf(sum_asq * 0.25f);
  float v = f3dot(c0, d2) * (1.0f / 6.0f);
  float r = sqrtf(arms);
  float den = r * r * r * perfect;
  Q32 out;
  out.q = v / den;
  // the triple product is off by at most 64 eps |d0||d1||d2|; each face
  // area by 12 eps of the square of the longest edge, so the denominator by
  // 24 eps lmax^2 / A_rms relative; the divisions and roots add 32 eps
  float n0 = f3dot(d0, d0), n1 = f3dot(d1, d1), n2 = f3dot(d2, d2);
  float lmax2 = fmaxf(fmaxf(fmaxf(n0, n1), fmaxf(n2, f3dot(e12, e12))),
      fmaxf(f3dot(e13, e13), f3dot(e23, e23)));
  float eps = 5.9604645e-08f;
  out.err = 64.0f * eps * (sqrtf(n0) * sqrtf(n1) * sqrtf(n2) / 6.0f) / den +
      fabsf(out.q) * eps * (32.0f + 24.0f * lmax2 / arms) + 1e-30f;
  if (!(den > 0.0f) || !isfinite(out.q) || !isfinite(out.err)) out.err = __int_as_float(0x7f800000);
  return out;
}

// which side of `thr` the metric edge length |xb - xa| / ((ha + hb) / 2)
// lies on, from a single-precision estimate: +1 above, -1 below, 0 when the
// estimate is within 64 float epsilons (relative) of the threshold
__device__ inline int edge_ratio_side_f32(double const* xa, double const* xb, double ha,
    double hb, double thr)
{
  float3 d = make_float3((float)(xb[0] - xa[0]), (float)(xb[1] - xa[1]), (float)(xb[2] - xa[2]));
  float r = sqrtf(f3dot(d, d)) / (float)((ha + hb) / 2);
  float t = (float)thr, band = 64.0f * 5.9604645e-08f * t;
  if (!isfinite(r)) return 0;
  if (r > t + band) return 1;
  if (r < t - band) return -1;
  return 0;
}

// device counters of the filter: candidates rejected on the estimate,
// candidates recomputed in double, the largest |estimate - double| seen and
// the number of times that exceeded the bound
struct Fp32Stats {
  unsigned long long decided;
  unsigned long long rechecked;
  unsigned int max_err_bits;
  unsigned int bound_exceeded;
};

__device__ inline void fp32_note_error(Fp32Stats* st, Q32 e, double q64)
{
  float diff = fabsf((float)(q64 - (double)e.q));
  atomicMax(&st->max_err_bits, __float_as_uint(diff));
  if ((double)diff > (double)e.err) atomicAdd(&st->bound_exceeded, 1u);
}

// tet_quality (quality.hpp:68-89): Shewchuk's V / A_rms^(3/2), normalised
__host__ __device__ inline double tet_quality(double const (*x)[3], double perfect)
{
  double sum_asq = 0;
  double a;
  a = tri_area(x[0], x[1], x[2]);
  sum_asq += a * a;
  a = tri_area(x[1], x[0], x[3]);
  sum_asq += a * a;
  a = tri_area(x[2], x[1], x[3]);
  sum_asq += a * a;
  a = tri_area(x[0], x[2], x[3]);
  sum_asq += a * a;
  double arms = sqrt(sum_asq / 4.);
  double v = tet_volume(x);
  double r = sqrt(arms);
  double q = v / (r * r * r);
  return q / perfect;
}

// triangle_quality / triangle_xy_quality (quality.hpp:34-66)
__host__ __device__ inline double tri_quality(double const (*x)[3], int z_area,
    double perfect)
{
  double sum = 0;
  sum += sqdist3(x[0], x[1]);
  sum += sqdist3(x[1], x[2]);
  sum += sqdist3(x[2], x[0]);
  double lrms = sqrt(sum / 3);
  double a = z_area ? tri_z_area(x[0], x[1], x[2]) : tri_area(x[0], x[1], x[2]);
  double q = a / (lrms * lrms);
  return q / perfect;
}

// element_quality (quality.hpp:101-109) / entity_quality (:91-99)
__host__ __device__ inline double elem_quality(u32 dim, double const (*x)[3],
    int xy_tri)
{
  return dim == 3 ? tet_quality(x, perfect_tet_quality())
                  : tri_quality(x, xy_tri, perfect_tri_quality());
}

__device__ inline void load3(double const* __restrict__ c, u32 v, double* o)
{
  o[0] = c[v * 3 + 0];
  o[1] = c[v * 3 + 1];
  o[2] = c[v * 3 + 2];
}

// ---------------------------------------------------------------------------
// host-side device memory (stream-ordered pool)

void* dev_alloc(size_t bytes, cudaStream_t s);
void dev_free(void* p, cudaStream_t s);

template <class T>
T* dalloc(size_t n, cudaStream_t s)
{
  return static_cast<T*>(dev_alloc(n * sizeof(T), s));
}

// read one value back (synchronises the stream)
u32 read_u32(u32 const* d, cudaStream_t s);
double read_f64(double const* d, cudaStream_t s);

}  // namespace osh
