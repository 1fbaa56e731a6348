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

// Programmatic dependent launch. Every kernel of the library starts with
// pdl_wait(), which returns once the kernels before it on the stream have
// finished and their writes are visible (a no-op for a kernel launched
// without the attribute), and every launch goes through launch_kernel,
// which sets the attribute: the next kernel's blocks are scheduled while
// the previous kernel's last blocks drain, instead of after a full launch
// gap. The launches are the same kernels with the same arguments in the
// same order; OSH_B200_PDL=0 in the environment launches without the
// attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

bool pdl_enabled();

template <class... KArgs, class... Args>
cudaError_t launch_kernel(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
    cudaStream_t stream, Args&&... args)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

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
// blocks of `block` threads covering n threads (at least one block)
inline u32 grid_for(u64 n, u32 block) { return n ? ceil_div(n, block) : 1; }

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

// Single-precision filter for quality and edge-length decisions.
//
// Each estimate comes with a rigorous bound on its distance from the value
// the double path computes, so a decision taken on the estimate is the
// double path's decision. The derivation (standard rounding-error analysis,
// u = 2^-24, gamma_n = n u / (1 - n u), no fused multiply-add since every
// unit is built with -fmad=false, IEEE float division and square root):
//
//  * inputs: d_k = fl32(fl64(x_k - x_0)) differs from the exact difference
//    D_k by a factor (1 + a), |a| <= u + 2^-53 + 2^-77, per component;
//  * volume: the triple product fl(fl(d0 x d1) . d2) is within
//    gamma_5 Pi(d) of det(d0, d1, d2), where Pi is the sum of the absolute
//    values of the six terms of the determinant, and det(d) within
//    3.0002 u Pi(d) of det(D); Pi(d) <= sqrt(2) |d0||d1||d2|, and |d_k| <=
//    sqrt(n_k)(1 + 1.51 u) for the computed squared lengths n_k, so
//    |V6 - det(D)| <= 12 u sqrt(n0 n1 n2);
//  * faces: each cross product c_i (of two edge vectors, formed from the
//    d_k with at most one more subtraction) is within 8.85 u lmax^2 of the
//    exact one (rounding of the cross product: gamma_2 sqrt(2) |a||b|;
//    edge vectors off by at most 3.0001 u lmax), and lmax^2 <= (1 + 9.01 u)
//    times the computed largest squared edge length lmax2: eps = 9 u lmax2;
//  * the sum S of the four |c_i|^2 (a sum of non-negative terms: gamma_6)
//    is within T = 7 u S + 4 eps sqrt(S) + 4 eps^2 of the exact one
//    (| |c|^2 - |C|^2 | <= |c - C| (2 |c| + |c - C|), sum |c_i| <= 2 sqrt(S));
//    delta = T / S;
//  * the denominator (S/16)^(3/4) 6 perfect, formed by two square roots,
//    three products and the rounded constant 6 perfect, is within a factor
//    1 +- rho_den of the exact one, rho_den = (delta + 9 u)(1 + 10 u), using
//    (1 + delta)^(3/4) <= 1 + delta and (1 - delta)^(3/4) >= 1 - delta;
//  * the quotient: with rho = rho_den (1 + 2u) + u and
//    E = 13 u sqrt(n0 n1 n2) / den, |q - q_exact| <= (rho |q| + E) / (1 - rho);
//  * the double path (the same operations with unit roundoff 2^-53 and
//    constants at most 1.2 times these) is within 2^-27 of that bound of
//    q_exact, which the factor (1 + 2^-20) covers; 2^-60 covers underflow
//    of products (every edge is at least 2^-20 long by the guard below).
//
// The bound is evaluated with every sum and product rounded upward (and
// 1 - rho downward), and every quotient and root through div_up / sqrt_up,
// which return a value at least the exact one, so it is at least the real
// bound. It is +inf (no decision on the estimate) when lmax2 is outside
// [2^-40, 2^40], S or the denominator is below 2^-120, delta > 1/8,
// rho > 1/4, the bound exceeds 1, or anything is not finite.
struct Q32 {
  float q;    // estimate of tet_quality
  float err;  // bound on |estimate - tet_quality in double|; +inf when none
};

constexpr float F32_U = 5.9604644775390625e-08f;  // 2^-24

__device__ inline float3 f3sub(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ inline float3 f3cross(float3 a, float3 b)
{
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ inline float f3dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// 6 * perfect_tet_quality(), formed in double and rounded once to float
__host__ __device__ inline float tet_k6_f32() { return (float)(6.0 * perfect_tet_quality()); }

// Upper bounds of a quotient and a square root from fast operations (the
// bound needs no correctly rounded result, only one that is not below the
// exact value): __fdividef is within 2 ulp of a / b for b in [2^-126, 2^126]
// (CUDA math API), so a / b <= q (1 + 8u); sqrtf is correctly rounded, so
// sqrt(x) <= r (1 + 2u); the product is rounded upward. Callers keep b and x
// in range (their guards).
__device__ inline float div_up(float a, float b)
{
  return __fmul_ru(__fdividef(a, b), 1.0f + 8.0f * F32_U);
}
__device__ inline float sqrt_up(float x) { return __fmul_ru(sqrtf(x), 1.0f + 2.0f * F32_U); }

__device__ inline Q32 tet_quality_f32(double const (*x)[3], float k6)
{
  float3 d0 = make_float3((float)(x[1][0] - x[0][0]), (float)(x[1][1] - x[0][1]),
      (float)(x[1][2] - x[0][2]));
  float3 d1 = make_float3((float)(x[2][0] - x[0][0]), (float)(x[2][1] - x[0][1]),
      (float)(x[2][2] - x[0][2]));
  float3 d2 = make_float3((float)(x[3][0] - x[0][0]), (float)(x[3][1] - x[0][1]),
      (float)(x[3][2] - x[0][2]));
  float3 e12 = f3sub(d1, d0), e13 = f3sub(d2, d0), e23 = f3sub(d2, d1);
  // faces {0,1,2}, {1,0,3}, {2,1,3}, {0,2,3} as cross products of two edges
  float3 c0 = f3cross(d0, d1), c1 = f3cross(d0, e13), c2 = f3cross(e12, e23), c3 = f3cross(d1, d2);
  float s = f3dot(c0, c0) + f3dot(c1, c1);
  s = s + f3dot(c2, c2);
  s = s + f3dot(c3, c3);
  float arms = sqrtf(s * 0.0625f);
  float r = sqrtf(arms);
  float den = r * r * r * k6;
  float v6 = f3dot(c0, d2);
  Q32 out;
  out.q = v6 / den;
  out.err = __int_as_float(0x7f800000);
  float n0 = f3dot(d0, d0), n1 = f3dot(d1, d1), n2 = f3dot(d2, d2);
  float lmax2 = fmaxf(fmaxf(fmaxf(n0, n1), fmaxf(n2, f3dot(e12, e12))),
      fmaxf(f3dot(e13, e13), f3dot(e23, e23)));
  if (!(lmax2 >= 0x1p-40f && lmax2 <= 0x1p40f) || !(den >= 0x1p-120f) || !(s >= 0x1p-120f) ||
      !isfinite(out.q))
    return out;
  float const u = F32_U;
  float eps = __fmul_ru(9.0f * u, lmax2);
  float t = __fadd_ru(__fadd_ru(__fmul_ru(7.0f * u, s),
      __fmul_ru(__fmul_ru(4.0f, eps), sqrt_up(s))), __fmul_ru(__fmul_ru(4.0f, eps), eps));
  float delta = div_up(t, s);
  // (1 + 10u and 1 + 2u are floats; 1 + 9u and 1 + u are not)
  float rho = __fmul_ru(__fadd_ru(delta, 9.0f * u), 1.0f + 10.0f * u);
  rho = __fadd_ru(__fmul_ru(rho, 1.0f + 2.0f * u), u);
  float e = div_up(__fmul_ru(13.0f * u, sqrt_up(__fmul_ru(__fmul_ru(n0, n1), n2))), den);
  float b = div_up(__fadd_ru(__fmul_ru(rho, fabsf(out.q)), e), __fadd_rd(1.0f, -rho));
  b = __fadd_ru(__fmul_ru(b, 1.0f + 0x1p-20f), 0x1p-60f);
  if (delta <= 0.125f && rho <= 0.25f && b <= 1.0f) out.err = b;
  return out;
}

// bounds of the interval the double value lies in (rounded outward)
__device__ inline float q32_lo(Q32 e) { return __fadd_rd(e.q, -e.err); }
__device__ inline float q32_hi(Q32 e) { return __fadd_ru(e.q, e.err); }

// Which side of `thr` the metric edge length |xb - xa| / ((ha + hb) / 2),
// as the double path computes it, lies on, from a single-precision estimate:
// +1 above, -1 below, 0 undecided. The estimate (differences rounded to
// float, a float dot product, square root, the mean size rounded to float,
// one division) is within 5.5001 u relative of the exact ratio and the
// double path within 4.6 * 2^-53, so an estimate with est (1 - 6u) > thr
// (formed in double: the product's rounding costs 2^-53) is above for both,
// and est (1 + 6u) < thr below. Undecided when the squared length or the
// mean size is outside [2^-100, 2^100] or the estimate is not finite.
__device__ inline int edge_ratio_side_f32(double const* xa, double const* xb, double ha,
    double hb, double thr)
{
  float3 d = make_float3((float)(xb[0] - xa[0]), (float)(xb[1] - xa[1]), (float)(xb[2] - xa[2]));
  float s = f3dot(d, d);
  float hv = (float)((ha + hb) / 2);
  if (!(s >= 0x1p-100f && s <= 0x1p100f && hv >= 0x1p-100f && hv <= 0x1p100f)) return 0;
  float r = sqrtf(s) / hv;
  double const u = 0x1p-24;
  if ((double)r * (1.0 - 6.0 * u) > thr) return 1;
  if ((double)r * (1.0 + 6.0 * u) < thr) return -1;
  return 0;
}

// device counters of the filter. decided / rechecked: decisions taken on
// the estimate and candidates that needed double values; max_err_bits /
// bound_exceeded: the largest |estimate - double| among estimates whose
// double value was computed, and how many exceeded their bound. With
// `audit` set (by the host, for tests), every decision taken on the
// estimate is also taken in double: audited counts them, flips counts those
// the double path takes differently, checked counts the estimates compared
// with their double value (bound_exceeded then covers all of them).
struct Fp32Stats {
  unsigned long long decided;
  unsigned long long rechecked;
  unsigned int max_err_bits;
  unsigned int bound_exceeded;
  unsigned int audit;
  unsigned int pad;
  unsigned long long audited;
  unsigned long long flips;
  unsigned long long checked;
};

// one estimate against its double value; lanes of the calling warp that are
// active here aggregate before touching the counters
__device__ inline void fp32_note_error(Fp32Stats* st, Q32 e, double q64)
{
  double d = fabs(q64 - (double)e.q);
  float diff = __double2float_ru(d);
  bool over = d > (double)e.err;
  unsigned m = __activemask();
  unsigned lead = __ffs(m) - 1;
  unsigned mx = __reduce_max_sync(m, __float_as_uint(diff));
  unsigned nover = __popc(__ballot_sync(m, over));
  if ((threadIdx.x & 31) == lead) {
    atomicMax(&st->max_err_bits, mx);
    if (nover) atomicAdd(&st->bound_exceeded, nover);
    if (st->audit) atomicAdd(&st->checked, (unsigned long long)__popc(m));
  }
}

// per-warp sums of the decided / rechecked / audited / flipped flags; every
// lane of the warp must call it
__device__ inline void fp32_count_warp(Fp32Stats* st, bool decided, bool rechecked,
    bool audited, bool flipped)
{
  unsigned nd = __popc(__ballot_sync(0xffffffffu, decided));
  unsigned nr = __popc(__ballot_sync(0xffffffffu, rechecked));
  unsigned na = __popc(__ballot_sync(0xffffffffu, audited));
  unsigned nf = __popc(__ballot_sync(0xffffffffu, flipped));
  if ((threadIdx.x & 31) == 0) {
    if (nd) atomicAdd(&st->decided, (unsigned long long)nd);
    if (nr) atomicAdd(&st->rechecked, (unsigned long long)nr);
    if (na) atomicAdd(&st->audited, (unsigned long long)na);
    if (nf) atomicAdd(&st->flips, (unsigned long long)nf);
  }
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
