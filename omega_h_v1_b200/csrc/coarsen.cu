// Edge collapse on sm_100a: coarsen_by_size / coarsen_slivers
// (coarsen.cpp:13-70, coarsen_common.cpp:29-239, check_collapse_class.cpp,
// coarsen_qualities.cpp:12-79, collapses_to_verts.cpp, collapses_to_ents.cpp,
// coarsen_topology.cpp, coarsen_conserve.cpp, coarsen_fit.cpp, qr.cpp).
#include <algorithm>

#include "passes.hpp"

namespace osh {

__device__ inline u32 collapses(u32 code, u32 dir) { return (code >> dir) & 1u; }

// coarsen_size_code (coarsen.cpp:13-21) fused with measure_edge
__global__ void k_coarsen_size_codes(u32 ne, u32 const* __restrict__ voe,
    double const* __restrict__ x, double const* __restrict__ h, double size_floor,
    SegView sv, Fp32Stats* fs, u32* __restrict__ codes, u32* any)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  u32 c = 0;
  bool decided = false, rechecked = false, flipped = false;
  if (i < ne) {
    u32 a = voe[i * 2], b = voe[i * 2 + 1];
    double xa[3], xb[3];
    load3(x, a, xa);
    load3(x, b, xb);
    int r32 = fs ? edge_ratio_side_f32(xa, xb, h[a], h[b], size_floor) : 0;
    bool shorter = false;
    if (r32) {
      decided = true;
      shorter = r32 < 0;
    }
    if (!r32 || fs->audit) {
      rechecked = !r32;
      double len = sqrt(sqdist3(xb, xa));
      double want = (h[a] + h[b]) / 2;
      bool s64 = (len / want) < size_floor;
      flipped = r32 && s64 != shorter;
      shorter = s64;
    }
    c = (shorter && seg_acts(sv, a)) ? (u32)COLLAPSE_BOTH : (u32)DONT_COLLAPSE;
    codes[i] = c;
  }
  if (fs) fp32_count_warp(fs, decided, rechecked, decided && fs->audit, flipped);
  if (__any_sync(0xffffffffu, c) && (threadIdx.x & 31) == 0) atomicOr(any, 1u);
}

// coarsen_sliver_code (coarsen.cpp:38-49)
__global__ void k_coarsen_sliver_codes(u32 ne, u32 const* __restrict__ voe,
    u32 const* __restrict__ marked, u32* __restrict__ codes, u32* any)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  u32 c = 0;
  if (i < ne) {
    if (marked[voe[i * 2]]) c |= 1u;
    if (marked[voe[i * 2 + 1]]) c |= 2u;
    codes[i] = c;
  }
  if (__any_sync(0xffffffffu, c) && (threadIdx.x & 31) == 0) atomicOr(any, 1u);
}

// check_basic_edge_class (check_collapse_class.cpp:12-37)
__device__ inline u32 basic_class_code(u32 i, u32 code, u32 const* __restrict__ voe,
    u32 const* __restrict__ cdv, u32 const* __restrict__ cde)
{
  u32 c0 = cdv[voe[i * 2]], c1 = cdv[voe[i * 2 + 1]], ce = cde[i];
  if (c0 == c1) return c0 != ce ? (u32)DONT_COLLAPSE : code;
  if (collapses(code, 0) && c0 != ce) code &= ~1u;
  if (collapses(code, 1) && c1 != ce) code &= ~2u;
  return code;
}

// check_for_exposed_side (check_collapse_class.cpp:55-103), for the
// entities of dimension ed around edge i
struct ExposedSides {
  u32 ed;
  u32 const* u_offs;  // up(1, ed)
  u32 const* u_adj;
  u32 const* u_dirs;
  u32 const* vot;     // down(ed, 0)
  u32 const* sot;     // down(ed, ed - 1)
  u32 const* cdt;     // class_dim of dimension ed
  u32 const* cds;     // class_dim of dimension ed - 1
};

__device__ inline u32 exposed_sides_code(u32 i, u32 code, u32 const* __restrict__ voe,
    ExposedSides const& x)
{
  u32 const ed = x.ed, vpt = deg(ed, 0), spt = deg(ed, ed - 1);
  for (u32 j = x.u_offs[i]; j < x.u_offs[i + 1]; ++j) {
    u32 t = x.u_adj[j], dir = x.u_dirs[j];
    u32 tcd = x.cdt[t];
    for (u32 k = 0; k < 2; ++k) {
      if (!collapses(code, k)) continue;
      u32 va = voe[i * 2 + (1 - k)];
      for (u32 l = 0; l < 2; ++l) {
        u32 eev = canon(ed, 1, 0, dir, l);
        if (x.vot[(size_t)t * vpt + eev] == va) {
          u32 side = x.sot[(size_t)t * spt + opp(ed, 0, eev)];
          if (x.cds[side] != tcd) code &= ~(1u << k);
          break;
        }
      }
    }
  }
  return code;
}

// The class checks of every edge with a code (the basic check, then the
// exposed sides for faces, then for elements: nxs of them), the code
// written back, each edge's collapse qualities zeroed, and the edges still
// with a code listed (a warp's appends in one counter update): one launch
// for what were a kernel per check and one for the list
__global__ void k_coarsen_class_list(u32 ne, u32 const* __restrict__ voe,
    u32 const* __restrict__ cdv, u32 const* __restrict__ cde, ExposedSides xs0,
    ExposedSides xs1, u32 nxs, u32* __restrict__ codes, u32* __restrict__ list, u32* count,
    double2* __restrict__ q2)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  bool on = false;
  if (i < ne) {
    q2[i] = make_double2(0.0, 0.0);
    u32 code = codes[i];
    if (code != DONT_COLLAPSE) {
      code = basic_class_code(i, code, voe, cdv, cde);
      if (code != DONT_COLLAPSE && nxs > 0) code = exposed_sides_code(i, code, voe, xs0);
      if (code != DONT_COLLAPSE && nxs > 1) code = exposed_sides_code(i, code, voe, xs1);
      codes[i] = code;
    }
    on = code != 0;
  }
  u32 mask = __ballot_sync(0xffffffffu, on);
  if (!mask) return;
  u32 lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
  u32 base = 0;
  if (lane == leader) base = atomicAdd(count, (u32)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (on) list[base + __popc(mask & ((1u << lane) - 1u))] = i;
}

// coarsen_quality (coarsen_qualities.cpp:12-79): worst element of the cavity
// after collapsing each allowed direction. One warp per candidate edge (from
// a compact list): the lanes share the collapsing vertex's elements, so a
// few candidates with long rows no longer idle the other lanes of a warp.
// Each minimum is reduced as (value, position) pairs, so the value kept is
// the one the sequential loop keeps: the first in row order among equals
// (which decides the sign of a zero), with NaN never taken.
struct FirstMin {
  double v;
  u32 k;  // 0 = the loop's initial value, else 1 + position in the row
};

__device__ inline void first_min_add(FirstMin& m, double q, u32 k)
{
  if (q < m.v) {
    m.v = q;
    m.k = k;
  }
}

__device__ inline double warp_first_min(FirstMin m)
{
  for (int o = 16; o; o >>= 1) {
    double ov = __shfl_xor_sync(0xffffffffu, m.v, o);
    u32 ok = __shfl_xor_sync(0xffffffffu, m.k, o);
    if (ov < m.v || (ov == m.v && ok < m.k)) {
      m.v = ov;
      m.k = ok;
    }
  }
  return m.v;
}

__device__ inline float warp_minf(float v)
{
  for (int o = 16; o; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <u32 DIM>
__global__ void k_coarsen_quality(u32 const* __restrict__ list,
    u32 const* __restrict__ nlist, u32 const* __restrict__ voe1, u32 const* __restrict__ voe,
    u32 const* __restrict__ ev_offs, u32 const* __restrict__ ev,
    u32 const* __restrict__ ev_dirs, double const* __restrict__ x,
    double const* __restrict__ eq, double floor_q, SegView sv, Fp32Stats* fs,
    u32* __restrict__ codes, double* __restrict__ out, u32* any)
{
  pdl_wait();
  constexpr u32 dim = DIM;  // element dimension: corner loops unroll into registers
  u32 lane = threadIdx.x & 31;
  u32 n = *nlist;
  constexpr u32 vpe = deg(dim, 0);
  double const perfect = dim == 3 ? perfect_tet_quality() : perfect_tri_quality();
  bool const use32 = fs && dim == 3;
  float const k6 = tet_k6_f32();
  for (u32 w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n;
       w += (gridDim.x * blockDim.x) >> 5) {
    u32 i = list[w];
    u32 code = codes[i];
    double const fq = seg_floor(sv, voe1[i * 2], floor_q);
    for (u32 j = 0; j < 2; ++j) {
      if (!collapses(code, j)) continue;
      u32 col = voe1[i * 2 + j], gen = voe1[i * 2 + 1 - j];
      u32 f = ev_offs[col], e = ev_offs[col + 1];
      double ex[4][3];
      load3(x, gen, ex[vpe - 1]);
      FirstMin om{1.0, 0};
      if (eq)
        for (u32 k = f + lane; k < e; k += 32) first_min_add(om, eq[ev[k]], k - f + 1);
      double old_minq = warp_first_min(om);
      // with the filter: the cavity's estimates first; the direction is
      // rejected on them when the worst element is surely below the floor or
      // surely no better than before; otherwise only the elements whose
      // lower bound reaches the lowest upper bound (they alone can hold the
      // minimum) are computed in double
      bool rejected32 = false, filtered = false;
      unsigned long long need = 0;   // this lane's elements, by visit index
      bool all = true;
      if (use32) {
        float upper = 1.0f;
        all = (e - f) > 64 * 32;
        u32 c = 0;
        for (u32 k = f + lane; k < e; k += 32, ++c) {
          u32 const* ve = voe + (size_t)ev[k] * vpe;
          bool adjacent = false;
          for (u32 l = 0; l < vpe; ++l) adjacent = adjacent || ve[l] == gen;
          if (adjacent) continue;
          u32 base = opp(dim, 0, ev_dirs[k]);
          for (u32 l = 0; l + 1 < vpe; ++l) load3(x, ve[canon(dim, dim - 1, 0, base, l)], ex[l]);
          Q32 q = tet_quality_f32(ex, k6);
          upper = fminf(upper, q32_hi(q));
          if (!all && q32_lo(q) <= upper) need |= 1ull << c;
        }
        upper = warp_minf(upper);
        filtered = true;
        rejected32 = (double)upper < fq || (eq && (double)upper <= old_minq);
        if (lane == 0) {
          if (rejected32)
            atomicAdd(&fs->decided, 1ull);
          else
            atomicAdd(&fs->rechecked, 1ull);
        }
      }
      double minq = 1.0;
      if (!rejected32) {
        FirstMin mm{1.0, 0};
        u32 c = 0;
        for (u32 k = f + lane; k < e; k += 32, ++c) {
          if (filtered && !all && !((need >> c) & 1ull)) continue;
          u32 const* ve = voe + (size_t)ev[k] * vpe;
          bool adjacent = false;
          for (u32 l = 0; l < vpe; ++l) adjacent = adjacent || ve[l] == gen;
          if (adjacent) continue;
          u32 base = opp(dim, 0, ev_dirs[k]);
          for (u32 l = 0; l + 1 < vpe; ++l) load3(x, ve[canon(dim, dim - 1, 0, base, l)], ex[l]);
          double q = dim == 3 ? tet_quality(ex, perfect) : tri_quality(ex, 1, perfect);
          if (filtered && fs->audit) fp32_note_error(fs, tet_quality_f32(ex, k6), q);
          first_min_add(mm, q, k - f + 1);
        }
        minq = warp_first_min(mm);
      }
      bool drop = rejected32 || minq < fq || (eq && minq <= old_minq);
      if (filtered && fs->audit) {
        // the double path's result over the whole cavity, and every
        // estimate against its double value
        FirstMin m64{1.0, 0};
        for (u32 k = f + lane; k < e; k += 32) {
          u32 const* ve = voe + (size_t)ev[k] * vpe;
          bool adjacent = false;
          for (u32 l = 0; l < vpe; ++l) adjacent = adjacent || ve[l] == gen;
          if (adjacent) continue;
          u32 base = opp(dim, 0, ev_dirs[k]);
          for (u32 l = 0; l + 1 < vpe; ++l) load3(x, ve[canon(dim, dim - 1, 0, base, l)], ex[l]);
          double q = tet_quality(ex, perfect);
          fp32_note_error(fs, tet_quality_f32(ex, k6), q);
          first_min_add(m64, q, k - f + 1);
        }
        double q64 = warp_first_min(m64);
        bool drop64 = q64 < fq || (eq && q64 <= old_minq);
        bool flip = drop64 != drop || (!drop && q64 != minq);
        if (lane == 0) {
          atomicAdd(&fs->audited, 1ull);
          if (flip) atomicAdd(&fs->flips, 1ull);
        }
      }
      if (drop)
        code &= ~(1u << j);
      else if (lane == 0)
        out[i * 2 + j] = minq;
    }
    if (lane == 0) {
      codes[i] = code;
      if (code != DONT_COLLAPSE) atomicOr(any, 1u);
    }
  }
}

// the candidate edges listed (a warp's candidates take consecutive slots,
// warps in any order) and every edge's two collapse qualities zeroed (the
// quality kernel writes the kept ones)
// collapse_to_vert (collapses_to_verts.cpp:13-42)
__global__ void k_collapses_to_verts(u32 nv, u32 const* __restrict__ ue_offs,
    u32 const* __restrict__ ue, u32 const* __restrict__ ue_dirs,
    u32 const* __restrict__ codes, double const* __restrict__ q2, u32* __restrict__ cand,
    double* __restrict__ colq)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  double maxq = 0;
  u32 c = 0;
  for (u32 j = ue_offs[i]; j < ue_offs[i + 1]; ++j) {
    u32 e = ue[j], d = ue_dirs[j];
    if (!collapses(codes[e], d)) continue;
    double q = q2[e * 2 + d];
    if (!c) {
      c = 1;
      maxq = q;
    } else if (q > maxq) {
      maxq = q;
    }
  }
  cand[i] = c;
  colq[i] = c ? maxq : 0.0;
}

// vertex_dest (collapses_to_verts.cpp:72-105): first edge in upward order
// whose collapse quality equals the vertex's best
__global__ void k_vertex_dest(u32 nv, u32 const* __restrict__ ue_offs,
    u32 const* __restrict__ ue, u32 const* __restrict__ ue_dirs,
    u32 const* __restrict__ voe1, u32 const* __restrict__ ind,
    double const* __restrict__ colq, u32 const* __restrict__ codes,
    double const* __restrict__ q2, u32* __restrict__ gen_vert)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  u32 g = INV;
  if (ind[i]) {
    double maxq = colq[i];
    if (maxq == 1e10) maxq = -1e10;
    for (u32 j = ue_offs[i]; j < ue_offs[i + 1]; ++j) {
      u32 e = ue[j], d = ue_dirs[j];
      if (!collapses(codes[e], d)) continue;
      double q = q2[e * 2 + d];
      if (q == 1e10) q = -1e10;
      if (q == maxq) {
        g = voe1[e * 2 + (1 - d)];
        break;
      }
    }
  }
  gen_vert[i] = g;
}

// The two vertex kernels with a group of VG lanes per vertex row (rows of
// about 13.5 edges; VG is the tuning table's vert_group): lane l takes the
// row's entries l, l + VG, ..., and shuffles within the group combine the
// lanes' results. The best collapse keeps the first entry (in upward order)
// of greatest quality, as the reference's loop does, so lanes combine
// (quality, position) pairs; the destination is the first entry whose
// quality equals the best.

template <u32 VG>
__global__ void k_collapses_to_verts_grouped(u32 nv, u32 const* __restrict__ ue_offs,
    u32 const* __restrict__ ue, u32 const* __restrict__ ue_dirs,
    u32 const* __restrict__ codes, double const* __restrict__ q2, u32* __restrict__ cand,
    double* __restrict__ colq)
{
  pdl_wait();
  u32 const t = blockIdx.x * blockDim.x + threadIdx.x;
  u32 const i = t / VG, lg = t % VG;
  if (i >= nv) return;  // a group shares i: it leaves together
  u32 const gbase = (threadIdx.x & 31) & ~(VG - 1);
  u32 const gmask = ((1u << VG) - 1u) << gbase;
  double maxq = 0;
  u32 pos = INV;  // position of the lane's best entry; INV: no collapse seen
  for (u32 j = ue_offs[i] + lg; j < ue_offs[i + 1]; j += VG) {
    u32 e = ue[j], d = ue_dirs[j];
    if (!collapses(codes[e], d)) continue;
    double q = q2[e * 2 + d];
    if (pos == INV || q > maxq) {
      maxq = q;
      pos = j;
    }
  }
  for (u32 o = VG / 2; o; o >>= 1) {
    double oq = __shfl_xor_sync(gmask, maxq, o);
    u32 op = __shfl_xor_sync(gmask, pos, o);
    if (op != INV && (pos == INV || oq > maxq || (oq == maxq && op < pos))) {
      maxq = oq;
      pos = op;
    }
  }
  if (lg == 0) {
    cand[i] = pos != INV;
    colq[i] = pos != INV ? maxq : 0.0;
  }
}

template <u32 VG>
__global__ void k_vertex_dest_grouped(u32 nv, u32 const* __restrict__ ue_offs,
    u32 const* __restrict__ ue, u32 const* __restrict__ ue_dirs,
    u32 const* __restrict__ voe1, u32 const* __restrict__ ind,
    double const* __restrict__ colq, u32 const* __restrict__ codes,
    double const* __restrict__ q2, u32* __restrict__ gen_vert)
{
  pdl_wait();
  u32 const t = blockIdx.x * blockDim.x + threadIdx.x;
  u32 const i = t / VG, lg = t % VG;
  if (i >= nv) return;
  u32 const gbase = (threadIdx.x & 31) & ~(VG - 1);
  u32 const gmask = ((1u << VG) - 1u) << gbase;
  if (!ind[i]) {
    if (lg == 0) gen_vert[i] = INV;
    return;
  }
  double maxq = colq[i];
  if (maxq == 1e10) maxq = -1e10;
  u32 first = INV;
  for (u32 j = ue_offs[i] + lg; j < ue_offs[i + 1]; j += VG) {
    u32 e = ue[j], d = ue_dirs[j];
    if (!collapses(codes[e], d)) continue;
    double q = q2[e * 2 + d];
    if (q == 1e10) q = -1e10;
    if (q == maxq) {
      first = j;
      break;
    }
  }
  for (u32 o = VG / 2; o; o >>= 1) first = min(first, __shfl_xor_sync(gmask, first, o));
  if (lg == 0) {
    u32 g = INV;
    if (first != INV) g = voe1[ue[first] * 2 + (1 - ue_dirs[first])];
    gen_vert[i] = g;
  }
}

// collapse_to_ent (collapses_to_ents.cpp:11-64)
// (ED: the entities' dimension at compile time, so the loads of all their
// vertices are issued before any is used)
// (fused_ents / fused_sides: the entities / sides a collapse fuses, marked
// with the stamps ents_gen / sides_gen of the stream's kept marks)
template <u32 ED>
__global__ void k_collapse_to_ent(u32 n, u32 const* __restrict__ voe,
    u32 const* __restrict__ soe, u32 const* __restrict__ gen_offs_v,
    u32 const* __restrict__ gen_vert_v, u32 const* __restrict__ fused_ents, u32 ents_gen,
    u32* __restrict__ is_same, u32* __restrict__ fused_sides, u32 sides_gen,
    u32* __restrict__ will_gen, u32* __restrict__ gen_vert, u32* __restrict__ gen_dir)
{
  pdl_wait();
  constexpr u32 VPE = ED + 1, SPE = ED + 1;
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 v[VPE], a[VPE], b[VPE];
#pragma unroll
  for (u32 j = 0; j < VPE; ++j) v[j] = voe[(size_t)i * VPE + j];
#pragma unroll
  for (u32 j = 0; j < VPE; ++j) {
    a[j] = gen_offs_v[v[j]];
    b[j] = gen_offs_v[v[j] + 1];
  }
  u32 col = INV, dir = INV;
#pragma unroll
  for (u32 j = 0; j < VPE; ++j)
    if (a[j] != b[j]) {  // the last collapsing vertex in local order wins
      col = v[j];
      dir = j;
    }
  u32 wg = 0;
  if (dir == INV) {
    is_same[i] = 1;
    will_gen[i] = 0;
    return;
  }
  is_same[i] = 0;
  u32 gv = gen_vert_v[col], gd = INV;
#pragma unroll
  for (u32 j = 0; j < VPE; ++j)
    if (v[j] == gv) gd = j;
  if (gd != INV) {
    fused_sides[soe[(size_t)i * SPE + opp(ED, 0, gd)]] = sides_gen;
  } else if (!(fused_ents && fused_ents[i] == ents_gen)) {
    wg = 1;
    gen_vert[i] = gv;
    gen_dir[i] = dir;
  }
  will_gen[i] = wg;
}

// coarsen_elem (coarsen_topology.cpp:9-34) writing straight into the new
// connectivity after the same entities, with remap_conn applied
// (coarsen_common.cpp:29-33)
// a thread per generating entity, from their list in order (the t-th
// generates the t-th product)
__global__ void k_coarsen_topology(u32 ed, u32 ngen, u32 const* __restrict__ gen_list,
    u32 const* __restrict__ voe, u32 const* __restrict__ gen_vert,
    u32 const* __restrict__ gen_dir, u32 const* __restrict__ same_v,
    u32* __restrict__ out)
{
  pdl_wait();
  u32 t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ngen) return;
  u32 const i = gen_list[t];
  u32 vpe = deg(ed, 0);
  u32* o = out + (size_t)t * vpe;
  u32 b = opp(ed, 0, gen_dir[i]);
  for (u32 j = 0; j + 1 < vpe; ++j)
    o[j] = same_v[voe[(size_t)i * vpe + canon(ed, ed - 1, 0, b, j)]];
  o[vpe - 1] = same_v[gen_vert[i]];
}

// expansion of the surviving entities' vertices, renumbered
template <u32 VPE>
__global__ void k_same_conn(u32 n, u32 const* __restrict__ voe, u32 const* __restrict__ same_e,
    u32 const* __restrict__ same_v, u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || same_e[i] == same_e[i + 1]) return;
  u32 o = same_e[i], v[VPE];
#pragma unroll
  for (u32 j = 0; j < VPE; ++j) v[j] = voe[(size_t)i * VPE + j];
#pragma unroll
  for (u32 j = 0; j < VPE; ++j) out[(size_t)o * VPE + j] = same_v[v[j]];
}

// coarsen_conserve_cavity (coarsen_conserve.cpp:15-55)
__global__ void k_coarsen_conserve(u32 nv, u32 nc, u32 nsame,
    u32 const* __restrict__ gen_offs_v, u32 const* __restrict__ gen_offs_e,
    u32 const* __restrict__ ev_offs, u32 const* __restrict__ ev,
    double const* __restrict__ in, double const* __restrict__ sizes,
    double* __restrict__ gen)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv || gen_offs_v[i] == gen_offs_v[i + 1]) return;
  u32 f = ev_offs[i], e = ev_offs[i + 1];
  double sum[MAX_NCOMPS];
  for (u32 c = 0; c < nc; ++c) sum[c] = 0;
  for (u32 j = f; j < e; ++j)
    for (u32 c = 0; c < nc; ++c) sum[c] = sum[c] + in[(size_t)ev[j] * nc + c];
  double cav = 0;
  for (u32 j = f; j < e; ++j) {
    u32 el = ev[j];
    if (gen_offs_e[el] == gen_offs_e[el + 1]) continue;
    cav += sizes[gen_offs_e[el] + nsame];
  }
  for (u32 j = f; j < e; ++j) {
    u32 el = ev[j];
    if (gen_offs_e[el] == gen_offs_e[el + 1]) continue;
    u32 ge = gen_offs_e[el];
    double sc = sizes[ge + nsame] / cav;
    for (u32 c = 0; c < nc; ++c) gen[(size_t)ge * nc + c] = sum[c] * sc;
  }
}

// ---- least-squares linear fit (qr.cpp:42-205, coarsen_fit.cpp:17-86) ----
__device__ inline double sgn(double x) { return (x < 0) ? -1 : 1; }

__device__ u32 qr_decomp2(double (*a)[4], double (*q)[MAX_PTS], double (*r)[4], u32 npts)
{
  for (u32 i = 0; i < npts; ++i)
    for (u32 j = 0; j < 4; ++j) r[i][j] = a[i][j];
  for (u32 i = 0; i < npts; ++i)
    for (u32 j = 0; j < npts; ++j) q[i][j] = (double)(i == j);
  double v[MAX_PTS];
  for (u32 i = 0; i < MAX_PTS; ++i) v[i] = 0;
  u32 rank = 0;
  for (u32 k = 0; k < 4; ++k) {
    // get_reflector2
    double cnorm = 0;
    for (u32 i = k; i < npts; ++i) cnorm += r[i][k] * r[i][k];
    cnorm = sqrt(cnorm);
    if (cnorm < 1e-6) continue;
    for (u32 i = 0; i < k; ++i) v[i] = 0;
    for (u32 i = k; i < npts; ++i) v[i] = r[i][k];
    v[k] += sgn(r[k][k]) * cnorm;
    double rnorm = 0;
    for (u32 i = k; i < npts; ++i) rnorm += v[i] * v[i];
    rnorm = sqrt(rnorm);
    for (u32 i = k; i < npts; ++i) v[i] /= rnorm;
    // reflect_columns2 / reflect_rows2
    for (u32 j = 0; j < 4; ++j) {
      double dot = 0;
      for (u32 i = k; i < npts; ++i) dot += r[i][j] * v[i];
      for (u32 i = k; i < npts; ++i) r[i][j] -= 2 * dot * v[i];
    }
    for (u32 i = 0; i < npts; ++i) {
      double dot = 0;
      for (u32 j = k; j < npts; ++j) dot += q[i][j] * v[j];
      for (u32 j = k; j < npts; ++j) q[i][j] -= 2 * dot * v[j];
    }
    ++rank;
  }
  return rank;
}

__device__ void qr_solve2(double (*q)[MAX_PTS], double (*r)[4], double const* b, u32 npts,
    double* xo)
{
  double y[4];
  for (u32 i = 0; i < 4; ++i) {
    y[i] = 0;
    for (u32 j = 0; j < npts; ++j) y[i] += q[j][i] * b[j];
  }
  for (u32 ii = 0; ii < 4; ++ii) {
    u32 i = 4 - ii - 1;
    xo[i] = y[i];
    for (u32 j = i + 1; j < 4; ++j) xo[i] -= r[i][j] * xo[j];
    xo[i] /= r[i][i];
  }
}

__global__ void k_coarsen_fit(u32 nv, u32 nc, u32 nsame, u32 const* __restrict__ gen_offs_v,
    u32 const* __restrict__ gen_offs_e, u32 const* __restrict__ ev_offs,
    u32 const* __restrict__ ev, double const* __restrict__ oldx,
    double const* __restrict__ newx, double const* __restrict__ in,
    double* __restrict__ gen)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv || gen_offs_v[i] == gen_offs_v[i + 1]) return;
  u32 f = ev_offs[i], e = ev_offs[i + 1];
  u32 npts = e - f;
  if (npts > MAX_PTS) npts = MAX_PTS;
  bool fit = npts >= 4;
  double q[MAX_PTS][MAX_PTS];
  double r[MAX_PTS][4];
  if (fit) {
    double a[MAX_PTS][4];
    for (u32 j = 0; j < npts; ++j) {
      u32 oe = ev[f + j];
      a[j][0] = 1.0;
      a[j][1] = oldx[oe * 3 + 0];
      a[j][2] = oldx[oe * 3 + 1];
      a[j][3] = oldx[oe * 3 + 2];
    }
    if (qr_decomp2(a, q, r, npts) < 4) fit = false;
  }
  for (u32 j = 0; j < nc; ++j) {
    double b[MAX_PTS], c[4], avg = 0;
    if (fit) {
      for (u32 k = 0; k < npts; ++k) b[k] = in[(size_t)ev[f + k] * nc + j];
      qr_solve2(q, r, b, npts, c);
    } else {
      avg = 0;
      for (u32 k = f; k < e; ++k) avg += in[(size_t)ev[k] * nc + j];
      avg /= (e - f);
    }
    for (u32 k = f; k < e; ++k) {
      u32 oe = ev[k];
      if (gen_offs_e[oe] == gen_offs_e[oe + 1]) continue;
      u32 ge = gen_offs_e[oe];
      if (fit) {
        double const* nx = newx + (size_t)(ge + nsame) * 3;
        double dd = 0;
        dd += c[1] * nx[0];
        dd += c[2] * nx[1];
        dd += c[3] * nx[2];
        gen[(size_t)ge * nc + j] = c[0] + dd;
      } else {
        gen[(size_t)ge * nc + j] = avg;
      }
    }
  }
}

static void coarsen_transfer(Mesh& m, Mesh& out, u32 const* gen_offs_v,
    u32 const* gen_offs_e, u32 const* same_e, u32 nsame, u32 ngen)
{
  cudaStream_t s = m.s;
  u32 dim = m.dim, nv = m.count(0), ne = m.count(dim);
  UpAdj const& ev = m.ask_up(0, dim);
  bool any_f64 = false, any_fit = false;
  for (auto const& t : m.tags[dim]) {
    if (t.type == T_F64) any_f64 = true;
    if (t.type == T_F64 && t.transfer == X_POINTWISE) any_fit = true;
  }
  if (any_f64) {
    double* sizes = out.element_sizes();
    for (auto const& t : m.tags[dim]) {
      if (t.type != T_F64 || t.transfer != X_CONSERVE) continue;
      u32 nc = t.ncomps;
      if (nc > MAX_NCOMPS) throw Failure(E_ARG, "conserved field wider than 32");
      double* data = dalloc<double>((size_t)(nsame + ngen) * nc, s);
      expand_scaled(t.data, same_e, 1, ne, nc, 8, data, s);
      if (nv) {
        CK(launch_kernel(k_coarsen_conserve, dim3(grid_for(nv)), dim3(BLOCK), 0, s, nv, nc, nsame, gen_offs_v,
            gen_offs_e, ev.offs, ev.adj, static_cast<double const*>(t.data), sizes,
            data + (size_t)nsame * nc));
        CK_LAUNCH();
      }
      out.add_tag(dim, T_F64, t.name.c_str(), nc, t.transfer, data);
    }
    dev_free(sizes, s);
  }
  if (!any_fit) return;
  if (!m.find_tag(dim, "coordinates")) interp_coords_to_elems(m);
  interp_coords_to_elems(out);
  double const* oldx = static_cast<double const*>(m.find_tag(dim, "coordinates")->data);
  double const* newx = static_cast<double const*>(out.find_tag(dim, "coordinates")->data);
  for (auto const& t : m.tags[dim]) {
    if (t.type != T_F64 || t.transfer != X_POINTWISE) continue;
    u32 nc = t.ncomps;
    double* data = dalloc<double>((size_t)(nsame + ngen) * nc, s);
    expand_scaled(t.data, same_e, 1, ne, nc, 8, data, s);
    if (nv) {
      CK(launch_kernel(k_coarsen_fit, dim3(ceil_div(nv, 128)), dim3(128), 0, s, nv, nc, nsame, gen_offs_v, gen_offs_e,
          ev.offs, ev.adj, oldx, newx, static_cast<double const*>(t.data),
          data + (size_t)nsame * nc));
      CK_LAUNCH();
    }
    out.add_tag(dim, T_F64, t.name.c_str(), nc, t.transfer, data);
  }
}

// check_coarsen_class + check_coarsen_quality + valid_collapses_to_verts +
// the vertex independent set (coarsen_common.cpp:109-189). codes is updated
// in place; returns false when no collapse survives.
struct CoarsenSel {
  double* q2 = nullptr;
  u32* cand = nullptr;
  double* colq = nullptr;
  u32* ind = nullptr;
  u32* gen_vert = nullptr;
  void free(cudaStream_t s)
  {
    dev_free(q2, s);
    dev_free(cand, s);
    dev_free(colq, s);
    dev_free(ind, s);
    dev_free(gen_vert, s);
  }
};

// deferred: no read-back here (the candidate flags and the set's outcome
// come back with coarsen_build's), so it always returns true
static bool coarsen_select(Mesh& m, u32* codes, double qual_floor, bool require_better,
    CoarsenSel& sel, u32* codes_class_out, u32* codes_qual_out, bool deferred = false)
{
  cudaStream_t s = m.s;
  u32 dim = m.dim, ne = m.count(1), nv = m.count(0);
  Tag* cdv = m.find_tag(0, "class_dim");
  Tag* cde = m.find_tag(1, "class_dim");
  if (!cdv || !cde) throw Failure(E_ARG, "coarsening needs class_dim on every dimension");
  u32 const* voe1 = m.ask_down(1, 0);
  ExposedSides xs[2] = {};
  u32 nxs = 0;
  for (u32 ed = 2; ed <= dim; ++ed) {
    UpAdj const& u = m.ask_up(1, ed, false);
    Tag* cdt = m.find_tag(ed, "class_dim");
    Tag* cds = m.find_tag(ed - 1, "class_dim");
    if (!cdt || !cds) throw Failure(E_ARG, "coarsening needs class_dim on every dimension");
    xs[nxs++] = ExposedSides{ed, u.offs, u.adj, u.dirs, m.ask_down(ed, 0),
        m.ask_down(ed, ed - 1), static_cast<u32 const*>(cdt->data),
        static_cast<u32 const*>(cds->data)};
  }
  // the class checks, the candidate edges listed, and the qualities of
  // their collapses; one read-back (mailbox slots 4 and 7) tells whether any
  // edge was a candidate and whether any collapse survived
  u32* clist = dalloc<u32>(ne ? ne : 1, s);
  sel.q2 = dalloc<double>((size_t)ne * 2, s);
  u32* any = m.mb->dev + 4;
  u32* ncand = m.mb->dev + 7;
  CK(cudaMemsetAsync(any, 0, 4 * sizeof(u32), s));  // slots 4-7
  if (ne) {
    CK(launch_kernel(k_coarsen_class_list, dim3(grid_for(ne)), dim3(BLOCK), 0, s, ne, voe1,
        static_cast<u32 const*>(cdv->data), static_cast<u32 const*>(cde->data), xs[0], xs[1],
        nxs, codes, clist, ncand, reinterpret_cast<double2*>(sel.q2)));
    CK_LAUNCH();
  }
  if (codes_class_out)
    CK(cudaMemcpyAsync(codes_class_out, codes, sizeof(u32) * ne, cudaMemcpyDeviceToDevice, s));
  if (codes_qual_out)
    CK(cudaMemcpyAsync(codes_qual_out, codes, sizeof(u32) * ne, cudaMemcpyDeviceToDevice, s));
  if (dim >= 2 && ne) {
    double const* eq = require_better ? m.qualities() : nullptr;
    UpAdj const& ev = m.ask_up(0, dim, false);
    double nel = m.counts[dim];
    PROBE(P_COARSEN_QUALITY, s, 4.0 * (nv + 1) + 8.0 * deg(dim, 0) * nel + 8.0 * ne +
        4.0 * deg(dim, 0) * nel + 24.0 * nv + 8.0 * ne + 16.0 * ne);
    // a warp per listed edge; the list's length is read on the device
    u32 const qb = tuned(TK_QUALITY_BLOCK);
    u32 blocks = (u32)std::min<u64>(ceil_div((u64)ne * 32, qb), 148u * 16u * 256u / qb);
    CK(launch_kernel(dim == 3 ? k_coarsen_quality<3> : k_coarsen_quality<2>, dim3(blocks),
        dim3(qb), 0, s, clist, ncand, voe1, m.ask_down(dim, 0),
        ev.offs, ev.adj, ev.dirs, m.coords(), eq, qual_floor, m.segview(),
        m.fp32_filter ? fp32_stats_dev() : nullptr, codes, sel.q2, any));
    CK_LAUNCH();
  }
  dev_free(clist, s);
  if (codes_qual_out)
    CK(cudaMemcpyAsync(codes_qual_out, codes, sizeof(u32) * ne, cudaMemcpyDeviceToDevice, s));
  if (!deferred) {
    m.mb->fetch(s, 8);
    if (!m.mb->host[7]) return false;
    // check_coarsen_quality (coarsen_common.cpp:139-180) ghosts a parallel
    // mesh and exchanges the collapse codes whatever it then finds
    m.ensure_ghosting(1);
    m.note_exchange(1);
    if (!m.mb->host[4]) return false;
  }
  UpAdj const& ue = m.ask_up(0, 1);
  sel.cand = dalloc<u32>(nv, s);
  sel.colq = dalloc<double>(nv, s);
  if (nv) {
    u32 const vg = tuned(TK_VERT_GROUP);
    auto k = vg == 4 ? k_collapses_to_verts_grouped<4>
           : vg == 16 ? k_collapses_to_verts_grouped<16> : k_collapses_to_verts_grouped<8>;
    CK(launch_kernel(k, dim3(grid_for((u64)nv * vg)), dim3(BLOCK), 0, s, nv, ue.offs, ue.adj,
        ue.dirs, codes, sel.q2, sel.cand, sel.colq));
    CK_LAUNCH();
  }
  sel.ind = find_indset(m, 0, sel.cand, sel.colq, !deferred);
  sel.gen_vert = dalloc<u32>(nv, s);
  if (nv) {
    u32 const vg = tuned(TK_VERT_GROUP);
    auto k = vg == 4 ? k_vertex_dest_grouped<4>
           : vg == 16 ? k_vertex_dest_grouped<16> : k_vertex_dest_grouped<8>;
    CK(launch_kernel(k, dim3(grid_for((u64)nv * vg)), dim3(BLOCK), 0, s, nv, ue.offs, ue.adj,
        ue.dirs, voe1, sel.ind, sel.colq, codes, sel.q2, sel.gen_vert));
    CK_LAUNCH();
  }
  return true;
}

// coarsen_interior + coarsen_all_ents (coarsen_common.cpp:35-219)
// deferred: the selection's flags and the set's outcome come back with the
// counts; with no collapse kept it frees what it made and returns false
static bool coarsen_build(Mesh& m, CoarsenSel const& sel, bool deferred)
{
  cudaStream_t s = m.s;
  u32 dim = m.dim, nv = m.count(0);
  u32* gen_offs_v = exscan_new(sel.ind, nv, s);
  // the surviving vertices' count lands in mailbox slot 22, read back with
  // the other dimensions' counts
  u32* same_v = dalloc<u32>((size_t)nv + 1, s);
  // the scans below are independent of one another and of the collapse
  // kernels after them: they run together in one launch after the loop
  ScanJob sj[7];
  u32 nsj = 0;
  sj[nsj++] = ScanJob{gen_offs_v, same_v, m.mb->dev + 22, nullptr, nv, 1};
  u32* scan_in[6] = {};
  u32 nscan_in = 0;
  u32* fused[4] = {nullptr, nullptr, nullptr, nullptr};  // the stream's kept marks
  u32 fgen[4] = {0, 0, 0, 0};
  u32* same_of[4] = {nullptr, nullptr, nullptr, nullptr};
  u32 nsame_of[4] = {0, 0, 0, 0};
  // the products and survivors of every dimension are counted first (the
  // fused sides pass from each dimension to the next on the device), their
  // totals landing in mailbox slots 16 + 2 (ed - 1) and 17 + 2 (ed - 1), so
  // one read-back serves all dimensions
  u32* gen_offs_of[4] = {nullptr, nullptr, nullptr, nullptr};
  u32* gen_list_of[4] = {nullptr, nullptr, nullptr, nullptr};  // the generating entities
  u32* gvert_of[4] = {nullptr, nullptr, nullptr, nullptr};
  u32* gdir_of[4] = {nullptr, nullptr, nullptr, nullptr};
  // each kept entity's new id, written by the survivors' scan for the
  // dimensions whose upward adjacency is carried
  u32* newid_of[4] = {nullptr, nullptr, nullptr, nullptr};
  for (u32 dd = 0; dd < dim; ++dd) {
    u32 ed = dim - dd;
    u32 n = m.count(ed), vpe = deg(ed, 0);
    u32 const* voe = m.ask_down(ed, 0);
    u32 const* soe = m.ask_down(ed, ed - 1);
    u32 nsides = m.count(ed - 1);
    fused[ed - 1] = stream_marks(KEPT_FUSED + ed - 1, nsides ? nsides : 1, s, &fgen[ed - 1]);
    u32* is_same = dalloc<u32>(n, s);
    u32* will_gen = dalloc<u32>(n, s);
    gvert_of[ed] = dalloc<u32>(n, s);
    gdir_of[ed] = dalloc<u32>(n, s);
    if (n) {
      PROBE(P_COLLAPSE_TO_ENT, s, 4.0 * (vpe + deg(ed, ed - 1)) * n + 8.0 * (nv + 1) +
          4.0 * n * 4 + 4.0 * nsides);
      auto k = ed == 1 ? k_collapse_to_ent<1> : ed == 2 ? k_collapse_to_ent<2>
                                                        : k_collapse_to_ent<3>;
      CK(launch_kernel(k, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, voe, soe, gen_offs_v,
          sel.gen_vert, fused[ed], fgen[ed], is_same, fused[ed - 1], fgen[ed - 1], will_gen,
          gvert_of[ed], gdir_of[ed]));
      CK_LAUNCH();
    }
    gen_offs_of[ed] = dalloc<u32>((size_t)n + 1, s);
    gen_list_of[ed] = dalloc<u32>(n ? n : 1, s);
    sj[nsj++] = ScanJob{will_gen, gen_offs_of[ed], m.mb->dev + 16 + 2 * (ed - 1), nullptr, n, 0,
        gen_list_of[ed]};
    if (carried_high(m, ed)) newid_of[ed] = dalloc<u32>(n ? n : 1, s);
    same_of[ed] = dalloc<u32>((size_t)n + 1, s);
    sj[nsj++] = ScanJob{is_same, same_of[ed], m.mb->dev + 17 + 2 * (ed - 1), newid_of[ed], n, 0};
    scan_in[nscan_in++] = will_gen;
    scan_in[nscan_in++] = is_same;
  }
  exscan_jobs(sj, nsj, s);
  for (u32 k = 0; k < nscan_in; ++k) dev_free(scan_in[k], s);
  m.mb->fetch(s, deferred ? INDSET_FETCH_SLOTS : 23);
  if (deferred) {
    auto abandon = [&] {
      for (u32 d = 0; d < 4; ++d) {
        dev_free(same_of[d], s);
        dev_free(gen_offs_of[d], s);
        dev_free(gen_list_of[d], s);
        dev_free(gvert_of[d], s);
        dev_free(gdir_of[d], s);
        dev_free(newid_of[d], s);
      }
      dev_free(same_v, s);
      dev_free(gen_offs_v, s);
    };
    try {
      indset_check(m);
    } catch (...) {
      abandon();
      throw;
    }
    if (!m.mb->host[7] || !m.mb->host[4]) {  // no candidate, or no collapse kept
      abandon();
      last_pass_stats().indset_rounds = 0;
      // check_coarsen_quality ghosts a parallel mesh and exchanges the
      // collapse codes once any edge was a candidate
      if (m.mb->host[7]) {
        m.ensure_ghosting(1);
        m.note_exchange(1);
      }
      return false;
    }
  }
  u32 nv_out = m.mb->host[22];
  last_pass_stats().nselected = nv - nv_out;
  Mesh* out = m.spawn();
  out->set_ents(0, nv_out, nullptr);
  // tags_subset (subset.cpp:15-43): every vertex tag survives (one launch)
  std::vector<ExpandJob> vjobs;
  for (auto const& t : m.tags[0]) {
    u32 esz = tag_esz(t.type);
    void* d = dev_alloc((size_t)nv_out * t.ncomps * esz, s);
    ExpandJob jb;
    jb.in = t.data;
    jb.offs = same_v;
    jb.out = d;
    jb.n = nv;
    jb.width = t.ncomps;
    jb.esz = esz;
    vjobs.push_back(jb);
    out->add_tag(0, t.type, t.name.c_str(), t.ncomps, t.transfer, d);
  }
  if (m.seg) {
    out->seg = dalloc<u32>(nv_out, s);
    ExpandJob jb;
    jb.in = m.seg;
    jb.offs = same_v;
    jb.out = out->seg;
    jb.n = nv;
    jb.width = 1;
    vjobs.push_back(jb);
  }
  expand_many(vjobs, s);
  if (m.parallel) inherit_globals(*out, 0);
  // every dimension's label copies launched together after the loop (the
  // generated lists and offsets they read are freed after that launch)
  std::vector<ExpandJob> copies;
  u32* free_after[8] = {};
  u32 nfree = 0;
  for (u32 dd = 0; dd < dim; ++dd) {
    u32 ed = dim - dd;
    u32 n = m.count(ed), vpe = deg(ed, 0);
    u32 const* voe = m.ask_down(ed, 0);
    u32 ngen = m.mb->host[16 + 2 * (ed - 1)], nsame = m.mb->host[17 + 2 * (ed - 1)];
    u32* gen_offs = gen_offs_of[ed];
    u32* same_e = same_of[ed];
    u32* gvert = gvert_of[ed];
    u32* gdir = gdir_of[ed];
    u32 nout = nsame + ngen;
    u32* conn = dalloc<u32>((size_t)nout * vpe, s);
    if (n) {
      auto k = vpe == 2 ? k_same_conn<2> : vpe == 3 ? k_same_conn<3> : k_same_conn<4>;
      CK(launch_kernel(k, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, voe, same_e, same_v, conn));
      CK_LAUNCH();
      if (ngen) {
        CK(launch_kernel(k_coarsen_topology, dim3(grid_for(ngen)), dim3(BLOCK), 0, s, ed, ngen,
            gen_list_of[ed], voe, gvert, gdir, same_v, conn + (size_t)nsame * vpe));
        CK_LAUNCH();
      }
    }
    dev_free(gvert, s);
    dev_free(gdir, s);
    out->set_ents(ed, nout, conn);
    // setup_coarsen (inherit.cpp:140-157)
    Doms d;
    d.ndoms[0] = n;
    d.offs[0] = same_e;
    d.ngen[0] = nsame;
    d.ndoms[ed] = n;
    d.offs[ed] = gen_offs;
    d.ngen[ed] = ngen;
    d.list[ed] = gen_list_of[ed];
    d.nlist[ed] = ngen;
    d.finish();
    inherit_class(m, *out, ed, d, nullptr, &copies);
    free_after[nfree++] = gen_list_of[ed];
    if (m.parallel) inherit_globals(*out, ed);
    if (ed == dim) coarsen_transfer(m, *out, gen_offs_v, gen_offs, same_e, nsame, ngen);
    free_after[nfree++] = gen_offs;
    nsame_of[ed] = nsame;
  }
  expand_many(copies, s);
  for (u32 k = 0; k < nfree; ++k) dev_free(free_after[k], s);
  same_of[0] = same_v;
  nsame_of[0] = nv_out;
  // downward adjacency of the survivors carries over; the products are searched
  carry_down_all(m, *out, same_of, nsame_of);
  carry_up_all(m, *out, same_of, nsame_of, newid_of);
  for (u32 h = 0; h <= dim; ++h) dev_free(newid_of[h], s);
  for (u32 d = 0; d < 4; ++d) {
    dev_free(same_of[d], s);
  }
  dev_free(gen_offs_v, s);
  m.overwrite(out);
  return true;
}

// The selection's flags and the set's outcome come back with the build's
// first read-back: two host waits fewer per pass. (A parallel mesh's
// ghosting state that depends on the flags is set after that read-back: a
// pass that changes the mesh replaces that state anyway.)
static bool coarsen_deferred(Mesh& m)
{
  return m.dim >= 2;
}

static u32 coarsen_common(Mesh& m, u32* codes, double qual_floor, bool require_better)
{
  CoarsenSel sel;
  bool ok = false;
  bool const deferred = coarsen_deferred(m);
  try {
    ok = coarsen_select(m, codes, qual_floor, require_better, sel, nullptr, nullptr, deferred);
    if (ok) {
      seg_tally(m, 0, sel.ind);
      ok = coarsen_build(m, sel, deferred);
    }
  } catch (...) {
    sel.free(m.s);
    throw;
  }
  sel.free(m.s);
  if (ok) last_pass_stats().elems_out = m.count(m.dim);
  return ok ? 1 : 0;
}

u32 coarsen_by_size(Mesh& m, double qual_floor, double size_floor)
{
  cudaStream_t s = m.s;
  PassStats& st = last_pass_stats();
  st = PassStats();
  st.op = 2;
  st.elems_in = m.count(m.dim);
  u32 ne = m.count(1);
  Tag* h = m.find_tag(0, "adapt_size");
  if (!h) throw Failure(E_ARG, "mesh has no adapt_size vertex field");
  u32* codes = dalloc<u32>(ne, s);
  // the codes kernel's "any code" flag (slot 5) is not read: with no code,
  // the candidate list of coarsen_select comes back empty in its one
  // read-back
  u32* any = m.mb->dev + 5;
  if (ne) {
    CK(launch_kernel(k_coarsen_size_codes, dim3(grid_for(ne)), dim3(BLOCK), 0, s, ne, m.ask_down(1, 0), m.coords(),
        static_cast<double const*>(h->data), size_floor, m.segview(),
        m.fp32_filter ? fp32_stats_dev() : nullptr, codes, any));
    CK_LAUNCH();
  }
  u32 r = 0;
  try {
    r = coarsen_common(m, codes, qual_floor, false);
  } catch (...) {
    dev_free(codes, s);
    throw;
  }
  dev_free(codes, s);
  return r;
}

u32 coarsen_slivers(Mesh& m, double qual_floor, u32 nlayers)
{
  cudaStream_t s = m.s;
  PassStats& st = last_pass_stats();
  st = PassStats();
  st.op = 4;
  st.elems_in = m.count(m.dim);
  u32 ne = m.count(1);
  // coarsen_slivers (coarsen.cpp:51-70) ghosts a parallel mesh; marking the
  // sliver layers exchanges element marks, marking their vertices vertex marks
  m.ensure_ghosting(1);
  u32* sl = mark_slivers(m, qual_floor, nlayers);
  if (nlayers) m.note_exchange(m.dim);
  u32* mv = mark_down(m, m.dim, 0, sl);
  m.note_exchange(0);
  dev_free(sl, s);
  u32* codes = dalloc<u32>(ne, s);
  u32* any = m.mb->dev + 5;  // not read (as in coarsen_by_size)
  if (ne) {
    CK(launch_kernel(k_coarsen_sliver_codes, dim3(grid_for(ne)), dim3(BLOCK), 0, s, ne, m.ask_down(1, 0), mv, codes, any));
    CK_LAUNCH();
  }
  dev_free(mv, s);
  u32 r = 0;
  try {
    r = coarsen_common(m, codes, 0.0, true);
  } catch (...) {
    dev_free(codes, s);
    throw;
  }
  dev_free(codes, s);
  return r;
}

u32 coarsen_sets(Mesh& m, double qual_floor, double size_floor, u32* codes_size,
    u32* codes_class, u32* codes_qual, double* quals2, u32* cand, double* col_qual,
    u32* indset, u32* gen_vert)
{
  cudaStream_t s = m.s;
  u32 ne = m.count(1), nv = m.count(0);
  Tag* h = m.find_tag(0, "adapt_size");
  if (!h) throw Failure(E_ARG, "mesh has no adapt_size vertex field");
  u32* any = m.mb->dev + 5;
  CK(cudaMemsetAsync(any, 0, sizeof(u32), s));
  CK(cudaMemsetAsync(quals2, 0, sizeof(double) * ne * 2, s));
  CK(cudaMemsetAsync(cand, 0, sizeof(u32) * nv, s));
  CK(cudaMemsetAsync(col_qual, 0, sizeof(double) * nv, s));
  CK(cudaMemsetAsync(indset, 0, sizeof(u32) * nv, s));
  CK(cudaMemsetAsync(gen_vert, 0xff, sizeof(u32) * nv, s));
  if (ne) {
    CK(launch_kernel(k_coarsen_size_codes, dim3(grid_for(ne)), dim3(BLOCK), 0, s, ne, m.ask_down(1, 0), m.coords(),
        static_cast<double const*>(h->data), size_floor, m.segview(),
        m.fp32_filter ? fp32_stats_dev() : nullptr, codes_size, any));
    CK_LAUNCH();
  }
  u32* codes = dalloc<u32>(ne, s);
  CK(cudaMemcpyAsync(codes, codes_size, sizeof(u32) * ne, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(codes_class, codes_size, sizeof(u32) * ne, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(codes_qual, codes_size, sizeof(u32) * ne, cudaMemcpyDeviceToDevice, s));
  CoarsenSel sel;
  bool ok = false;
  if (read_u32(any, s)) {
    ok = coarsen_select(m, codes, qual_floor, false, sel, codes_class, codes_qual);
    if (sel.q2) {
      // only the directions that still collapse carry a quality
      CK(cudaMemcpyAsync(quals2, sel.q2, sizeof(double) * ne * 2, cudaMemcpyDeviceToDevice, s));
    }
    if (ok) {
      CK(cudaMemcpyAsync(cand, sel.cand, sizeof(u32) * nv, cudaMemcpyDeviceToDevice, s));
      CK(cudaMemcpyAsync(col_qual, sel.colq, sizeof(double) * nv, cudaMemcpyDeviceToDevice, s));
      CK(cudaMemcpyAsync(indset, sel.ind, sizeof(u32) * nv, cudaMemcpyDeviceToDevice, s));
      CK(cudaMemcpyAsync(gen_vert, sel.gen_vert, sizeof(u32) * nv, cudaMemcpyDeviceToDevice, s));
    }
  }
  stream_sync(s);
  sel.free(s);
  dev_free(codes, s);
  return ok ? 1 : 0;
}

}  // namespace osh
