// Edge swapping of sliver cavities on sm_100a: swap_slivers
// (swap.cpp:27-154, swap_qualities.cpp:13-61, edge_ring.cpp:12-74,
// edge_swap.cpp:230-386, swap_topology.cpp:16-123, swap_conserve.cpp,
// swap_fit.cpp).
//
// The triangulation chosen for an edge in the quality kernel is stored and
// reused by the rebuild (the reference re-derives it with the same
// arithmetic, so the result is the same).
#include <cstring>
#include <mutex>

#include "passes.hpp"
#include "swap_tables.h"

namespace osh {

struct SwapTab {
  unsigned char ntri[8];
  unsigned char nmesh[8];
  unsigned char nint[8];
  unsigned char nuniq[8];
  unsigned char tri[8][42][5][3];
  unsigned char uniq[8][42][5];
  unsigned char iedge[8][42][4][2];
};

__constant__ SwapTab c_swap;

// Interior edges of each triangulation in the order the reference's own
// side derivation emits them (test_print_swap_edges.cpp:29-58): triangles in
// order, sides (0,1),(1,2),(2,0), keeping a side when its neighbour triangle
// has a larger index.
static void build_swap_tables(SwapTab& t)
{
  std::memset(&t, 0, sizeof(t));
  for (u32 n = 3; n <= MAX_EDGE_SWAP; ++n) {
    char const* p = polygon_triangulations[n];
    u32 nt = n - 2, nm = 0, nu = 0;
    unsigned char seen[64][3];
    while (*p) {
      for (u32 k = 0; k < nt; ++k) {
        for (u32 c = 0; c < 3; ++c) t.tri[n][nm][k][c] = (unsigned char)(p[c] - '0');
        p += 3;
        if (*p == '.') ++p;
        u32 a;
        for (a = 0; a < nu; ++a)
          if (!std::memcmp(seen[a], t.tri[n][nm][k], 3)) break;
        if (a == nu) std::memcpy(seen[nu++], t.tri[n][nm][k], 3);
        t.uniq[n][nm][k] = (unsigned char)a;
      }
      while (*p == ' ') ++p;
      ++nm;
    }
    t.ntri[n] = (unsigned char)nt;
    t.nmesh[n] = (unsigned char)nm;
    t.nuniq[n] = (unsigned char)nu;
    for (u32 mm = 0; mm < nm; ++mm) {
      u32 ni = 0;
      for (u32 k = 0; k < nt; ++k)
        for (u32 j = 0; j < 3; ++j) {
          u32 a = t.tri[n][mm][k][j], b = t.tri[n][mm][k][(j + 1) % 3];
          u32 nb = INV;
          for (u32 o = 0; o < nt && nb == INV; ++o) {
            if (o == k) continue;
            bool ha = false, hb = false;
            for (u32 c = 0; c < 3; ++c) {
              ha |= t.tri[n][mm][o][c] == a;
              hb |= t.tri[n][mm][o][c] == b;
            }
            if (ha && hb) nb = o;
          }
          if (nb != INV && k < nb) {
            t.iedge[n][mm][ni][0] = (unsigned char)a;
            t.iedge[n][mm][ni][1] = (unsigned char)b;
            ++ni;
          }
        }
      t.nint[n] = (unsigned char)ni;
    }
  }
}

static std::once_flag g_swap_once[64];

static void ensure_swap_tables()
{
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::call_once(g_swap_once[dev & 63], []() {
    SwapTab t;
    build_swap_tables(t);
    CK(cudaMemcpyToSymbol(c_swap, &t, sizeof(t)));
  });
}

// host access for tests
void swap_table_host(u32 rs, u32* ntri, u32* nmesh, u32* nint, u32* tris, u32* iedges)
{
  SwapTab t;
  build_swap_tables(t);
  *ntri = t.ntri[rs];
  *nmesh = t.nmesh[rs];
  *nint = t.nint[rs];
  for (u32 i = 0; i < t.nmesh[rs]; ++i) {
    for (u32 j = 0; j < t.ntri[rs]; ++j)
      for (u32 k = 0; k < 3; ++k) *tris++ = t.tri[rs][i][j][k];
    for (u32 j = 0; j < t.nint[rs]; ++j)
      for (u32 k = 0; k < 2; ++k) *iedges++ = t.iedge[rs][i][j][k];
  }
}

// find_edge_ring (edge_ring.cpp:12-74): the ring vertices of an edge, in the
// order that walks around it starting from its first upward tet
__device__ u32 find_edge_ring(u32 edge, u32 const* __restrict__ te_offs,
    u32 const* __restrict__ te, u32 const* __restrict__ te_dirs,
    u32 const* __restrict__ voe1, u32 const* __restrict__ vot, u32* ev, u32* rv)
{
  u32 f = te_offs[edge], e = te_offs[edge + 1];
  u32 rs = e - f;
  if (rs > MAX_EDGE_SWAP) return rs;
  ev[0] = voe1[edge * 2];
  ev[1] = voe1[edge * 2 + 1];
  u32 ta[MAX_EDGE_SWAP], tb[MAX_EDGE_SWAP];
  for (u32 i = 0; i < rs; ++i) {
    u32 t = te[f + i], d = te_dirs[f + i];
    u32 const* tv = vot + (size_t)t * 4;
    u32 align = (tv[tet_edge_vert(d, 0)] != ev[0]) ? 1u : 0u;
    u32 o = tet_opp_edge(d);
    ta[i] = tv[tet_edge_vert(o, align ^ 0u)];
    tb[i] = tv[tet_edge_vert(o, align ^ 1u)];
  }
  for (u32 i = 0; i + 1 < rs; ++i) {
    u32 j;
    for (j = i + 1; j < rs; ++j)
      if (ta[j] == tb[i]) break;
    if (j == rs) return INV;  // not a closed ring
    u32 xa = ta[j], xb = tb[j];
    ta[j] = ta[i + 1];
    tb[j] = tb[i + 1];
    ta[i + 1] = xa;
    tb[i + 1] = xb;
  }
  for (u32 i = 0; i < rs; ++i) rv[i] = ta[i];
  return rs;
}

// choose_edge_swap (edge_swap.cpp:230-280): best triangulation by its worst
// tet, first one wins ties; unique triangles are evaluated once
__device__ void choose_edge_swap(u32 rs, double const (*ex)[3], double const (*rx)[3],
    double perfect, u32* code_out, double* q_out)
{
  unsigned long long cached = 0;
  double cache[35];
  u32 code = INV;
  double best = -1;
  u32 nm = c_swap.nmesh[rs], nt = c_swap.ntri[rs];
  for (u32 i = 0; i < nm; ++i) {
    double mesh_minq = 1;
    for (u32 j = 0; j < nt; ++j) {
      u32 slot = c_swap.uniq[rs][i][j];
      if (!((cached >> slot) & 1ull)) {
        double tx[4][3];
        for (u32 k = 0; k < 3; ++k) {
          u32 r = c_swap.tri[rs][i][j][k];
          tx[k][0] = rx[r][0];
          tx[k][1] = rx[r][1];
          tx[k][2] = rx[r][2];
        }
        double tri_minq = 1;
        for (u32 k = 0; k < 2; ++k) {
          tx[3][0] = ex[1 - k][0];
          tx[3][1] = ex[1 - k][1];
          tx[3][2] = ex[1 - k][2];
          double q = tet_quality(tx, perfect);
          if (q < tri_minq) tri_minq = q;
          for (u32 c = 0; c < 3; ++c) {
            double tmp = tx[0][c];
            tx[0][c] = tx[1][c];
            tx[1][c] = tmp;
          }
        }
        cached |= 1ull << slot;
        cache[slot] = tri_minq;
      }
      double tq = cache[slot];
      if (tq < mesh_minq) mesh_minq = tq;
      if (mesh_minq < 0) break;
    }
    if (mesh_minq > best) {
      code = i;
      best = mesh_minq;
    }
  }
  *code_out = code;
  *q_out = best;
}

// Upper bound, from single-precision estimates, on the best triangulation's
// worst tet as choose_edge_swap would find it, valid whenever that value is
// positive (a triangulation it stops early on has a negative value). With
// `audit`, every estimate is also compared with its double value.
__device__ float best_swap_upper_f32(u32 rs, double const (*ex)[3], double const (*rx)[3],
    float k6, Fp32Stats* audit)
{
  float cache[35];
  unsigned long long cached = 0;
  float best = -1.0f;
  u32 nm = c_swap.nmesh[rs], nt = c_swap.ntri[rs];
  for (u32 i = 0; i < nm; ++i) {
    float mesh_upper = 1.0f;
    for (u32 j = 0; j < nt; ++j) {
      u32 slot = c_swap.uniq[rs][i][j];
      if (!((cached >> slot) & 1ull)) {
        double tx[4][3];
        for (u32 k = 0; k < 3; ++k) {
          u32 r = c_swap.tri[rs][i][j][k];
          tx[k][0] = rx[r][0];
          tx[k][1] = rx[r][1];
          tx[k][2] = rx[r][2];
        }
        float tri_upper = 1.0f;
        for (u32 k = 0; k < 2; ++k) {
          tx[3][0] = ex[1 - k][0];
          tx[3][1] = ex[1 - k][1];
          tx[3][2] = ex[1 - k][2];
          Q32 q = tet_quality_f32(tx, k6);
          if (audit) fp32_note_error(audit, q, tet_quality(tx, perfect_tet_quality()));
          tri_upper = fminf(tri_upper, q32_hi(q));
          for (u32 c = 0; c < 3; ++c) {
            double tmp = tx[0][c];
            tx[0][c] = tx[1][c];
            tx[1][c] = tmp;
          }
        }
        cached |= 1ull << slot;
        cache[slot] = tri_upper;
      }
      mesh_upper = fminf(mesh_upper, cache[slot]);
    }
    best = fmaxf(best, mesh_upper);
  }
  return best;
}

// unmark_boundary (mark.cpp:198-204)
__global__ void k_unmark_boundary(u32 n, u32 dim, u32 const* __restrict__ cd,
    u32* __restrict__ marked, u32* any)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  u32 keep = 0;
  if (i < n) {
    if (cd[i] != dim) marked[i] = 0;
    keep = marked[i];
  }
  if (__any_sync(0xffffffffu, keep) && (threadIdx.x & 31) == 0) atomicOr(any, 1u);
}

// swap_quality (swap_qualities.cpp:13-61)
__global__ void k_swap_quality(u32 ne, u32 const* __restrict__ te_offs,
    u32 const* __restrict__ te, u32 const* __restrict__ te_dirs,
    u32 const* __restrict__ voe1, u32 const* __restrict__ vot,
    double const* __restrict__ x, double const* __restrict__ eq, Fp32Stats* fs,
    u32* __restrict__ cand, double* __restrict__ quals, u32* __restrict__ ring_sizes,
    u32* __restrict__ codes, u32* any)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  u32 keep = 0;
  bool decided = false, rechecked = false, audited = false, flipped = false;
  if (i < ne && cand[i]) {
    double old_minq = 1;
    for (u32 j = te_offs[i]; j < te_offs[i + 1]; ++j)
      if (eq[te[j]] < old_minq) old_minq = eq[te[j]];
    u32 ev[2], rv[MAX_EDGE_SWAP];
    u32 rs = find_edge_ring(i, te_offs, te, te_dirs, voe1, vot, ev, rv);
    if (rs > MAX_EDGE_SWAP || rs < 3) {
      cand[i] = 0;
    } else {
      double ex[2][3], rx[MAX_EDGE_SWAP][3];
      load3(x, ev[0], ex[0]);
      load3(x, ev[1], ex[1]);
      for (u32 j = 0; j < rs; ++j) load3(x, rv[j], rx[j]);
      u32 code;
      double q = -1;
      // a swap is kept only if it beats old_minq; when old_minq is positive
      // an upper bound at or below it settles the rejection
      bool filtered = false;
      if (fs && old_minq > 0) {
        float ub = best_swap_upper_f32(rs, ex, rx, tet_k6_f32(), fs->audit ? fs : nullptr);
        if ((double)ub <= old_minq) {
          filtered = true;
          decided = true;
          if (fs->audit) {
            u32 c64;
            double q64;
            choose_edge_swap(rs, ex, rx, perfect_tet_quality(), &c64, &q64);
            audited = true;
            flipped = q64 > old_minq;
          }
        } else {
          rechecked = true;
        }
      }
      if (!filtered) choose_edge_swap(rs, ex, rx, perfect_tet_quality(), &code, &q);
      if (!filtered && q > old_minq) {
        quals[i] = q;
        ring_sizes[i] = rs;
        codes[i] = code;
        keep = 1;
      } else {
        cand[i] = 0;
      }
    }
  }
  if (i < ne && !keep) {  // every edge's goodness and ring size is written here
    quals[i] = 0.0;
    ring_sizes[i] = 0;
  }
  if (fs) fp32_count_warp(fs, decided, rechecked, audited, flipped);
  if (__any_sync(0xffffffffu, keep) && (threadIdx.x & 31) == 0) atomicOr(any, 1u);
}

__device__ inline u32 count_swap_ents(u32 rs, u32 dim)
{
  if (dim == 1) return c_swap.nint[rs];
  if (dim == 2) return c_swap.ntri[rs] + 2u * c_swap.nint[rs];
  return 2u * c_swap.ntri[rs];
}

__global__ void k_swap_counts(u32 ne, u32 dim, u32 const* __restrict__ ind,
    u32 const* __restrict__ rs, u32* __restrict__ cnt)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ne) cnt[i] = ind[i] ? count_swap_ents(rs[i], dim) : 0u;
}

// swap_cavity + get_swap_ents (swap_topology.cpp:42-71, edge_swap.cpp:282-373)
__global__ void k_swap_cavity(u32 ne, u32 dim, u32 const* __restrict__ ind,
    u32 const* __restrict__ codes, u32 const* __restrict__ gen_offs,
    u32 const* __restrict__ te_offs, u32 const* __restrict__ te,
    u32 const* __restrict__ te_dirs, u32 const* __restrict__ voe1,
    u32 const* __restrict__ vot, u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne || !ind[i]) return;
  u32 ev[2], rv[MAX_EDGE_SWAP];
  u32 rs = find_edge_ring(i, te_offs, te, te_dirs, voe1, vot, ev, rv);
  u32 code = codes[i];
  u32 vpe = deg(dim, 0);
  u32* o = out + (size_t)gen_offs[i] * vpe;
  u32 nt = c_swap.ntri[rs], ni = c_swap.nint[rs];
  if (dim == 1) {
    for (u32 k = 0; k < ni; ++k) {
      o[k * 2 + 0] = rv[c_swap.iedge[rs][code][k][0]];
      o[k * 2 + 1] = rv[c_swap.iedge[rs][code][k][1]];
    }
  } else if (dim == 2) {
    for (u32 k = 0; k < ni; ++k)
      for (u32 j = 0; j < 2; ++j) {
        o[k * 6 + j * 3 + 0] = rv[c_swap.iedge[rs][code][k][0]];
        o[k * 6 + j * 3 + 1] = rv[c_swap.iedge[rs][code][k][1]];
        o[k * 6 + j * 3 + 2] = ev[j];
      }
    o += ni * 6;
    for (u32 k = 0; k < nt; ++k)
      for (u32 j = 0; j < 3; ++j) o[k * 3 + j] = rv[c_swap.tri[rs][code][k][j]];
  } else {
    for (u32 k = 0; k < nt; ++k) {
      u32 tv[4];
      for (u32 j = 0; j < 3; ++j) tv[j] = rv[c_swap.tri[rs][code][k][j]];
      for (u32 j = 0; j < 2; ++j) {
        tv[3] = ev[1 - j];
        for (u32 c = 0; c < 4; ++c) *o++ = tv[c];
        u32 t = tv[0];
        tv[0] = tv[1];
        tv[1] = t;
      }
    }
  }
}

// entities not adjacent to a swapped edge survive (swap.cpp:39-43)
// (LPH edges per entity at compile time: their loads are issued together)
template <u32 LPH>
__global__ void k_swap_same(u32 n, u32 const* __restrict__ loh, u32 const* __restrict__ ind,
    u32* __restrict__ same)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 e[LPH], f[LPH];
#pragma unroll
  for (u32 j = 0; j < LPH; ++j) e[j] = loh ? loh[(size_t)i * LPH + j] : i;
#pragma unroll
  for (u32 j = 0; j < LPH; ++j) f[j] = ind[e[j]];
  u32 r = 1;
#pragma unroll
  for (u32 j = 0; j < LPH; ++j)
    if (f[j]) r = 0;
  same[i] = r;
}

// swap_conserve_cavity (swap_conserve.cpp:15-50)
__global__ void k_swap_conserve(u32 ne, u32 nc, u32 nsame, u32 const* __restrict__ gen_offs,
    u32 const* __restrict__ te_offs, u32 const* __restrict__ te,
    double const* __restrict__ sizes, double const* __restrict__ in,
    double* __restrict__ gen)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne || gen_offs[i] == gen_offs[i + 1]) return;
  double sum[MAX_NCOMPS];
  for (u32 c = 0; c < nc; ++c) sum[c] = 0;
  for (u32 j = te_offs[i]; j < te_offs[i + 1]; ++j)
    for (u32 c = 0; c < nc; ++c) sum[c] = sum[c] + in[(size_t)te[j] * nc + c];
  u32 f = gen_offs[i], e = gen_offs[i + 1];
  double cav = 0;
  for (u32 j = f; j < e; ++j) cav += sizes[nsame + j];
  for (u32 j = f; j < e; ++j) {
    double sc = sizes[nsame + j] / cav;
    for (u32 c = 0; c < nc; ++c) gen[(size_t)j * nc + c] = sum[c] * sc;
  }
}

// swap_fit_cavity (swap_fit.cpp:24-50): plain average over the old cavity
__global__ void k_swap_fit(u32 ne, u32 nc, u32 const* __restrict__ gen_offs,
    u32 const* __restrict__ te_offs, u32 const* __restrict__ te,
    double const* __restrict__ in, double* __restrict__ gen)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne || gen_offs[i] == gen_offs[i + 1]) return;
  u32 f = te_offs[i], e = te_offs[i + 1];
  for (u32 c = 0; c < nc; ++c) {
    double avg = 0;
    for (u32 k = f; k < e; ++k) avg += in[(size_t)te[k] * nc + c];
    avg /= (e - f);
    for (u32 g = gen_offs[i]; g < gen_offs[i + 1]; ++g) gen[(size_t)g * nc + c] = avg;
  }
}

struct SwapSel {
  u32* cand = nullptr;
  double* quals = nullptr;
  u32* rs = nullptr;
  u32* codes = nullptr;
  u32* ind = nullptr;
  void free(cudaStream_t s)
  {
    dev_free(cand, s);
    dev_free(quals, s);
    dev_free(rs, s);
    dev_free(codes, s);
    dev_free(ind, s);
  }
};

// marks through the independent set (swap_slivers + swap_common,
// swap.cpp:99-154); the optional outputs record each stage
// deferred: no read-back here (the "any swap kept" flag and the set's
// outcome come back with swap_build's)
static bool swap_select(Mesh& m, double gq, u32 nlayers, SwapSel& sel, u32* slivers_out,
    u32* cand_out, u32* interior_out, bool deferred = false)
{
  cudaStream_t s = m.s;
  ensure_swap_tables();
  u32 ne = m.count(1), nel = m.count(3);
  // swap_slivers (swap.cpp:180-196) ghosts a parallel mesh; marking the
  // sliver layers exchanges element marks, marking their edges edge marks
  m.ensure_ghosting(1);
  u32* sl = mark_slivers(m, gq, nlayers);
  if (nlayers) m.note_exchange(3);
  if (slivers_out)
    CK(cudaMemcpyAsync(slivers_out, sl, sizeof(u32) * nel, cudaMemcpyDeviceToDevice, s));
  sel.cand = mark_down(m, 3, 1, sl);
  m.note_exchange(1);
  dev_free(sl, s);
  if (cand_out)
    CK(cudaMemcpyAsync(cand_out, sel.cand, sizeof(u32) * ne, cudaMemcpyDeviceToDevice, s));
  if (!ne) return false;
  Tag* cd = m.find_tag(1, "class_dim");
  if (!cd) throw Failure(E_ARG, "swapping needs class_dim on edges");
  // no read-back between the stages: an edge that is no candidate (no
  // sliver, or on the boundary) is skipped by the quality kernel, whose
  // "any swap kept" flag (mailbox slot 6) is the one read
  u32* any = m.mb->dev + 6;
  CK(cudaMemsetAsync(m.mb->dev + 5, 0, 2 * sizeof(u32), s));  // slots 5-6
  CK(launch_kernel(k_unmark_boundary, dim3(grid_for(ne)), dim3(BLOCK), 0, s, ne, m.dim, static_cast<u32 const*>(cd->data),
      sel.cand, m.mb->dev + 5));
  CK_LAUNCH();
  if (interior_out)
    CK(cudaMemcpyAsync(interior_out, sel.cand, sizeof(u32) * ne, cudaMemcpyDeviceToDevice, s));
  sel.quals = dalloc<double>(ne, s);
  sel.rs = dalloc<u32>(ne, s);
  sel.codes = dalloc<u32>(ne, s);
  UpAdj const& te = m.ask_up(1, 3);
  double const* eq = m.qualities();
  PROBE(P_SWAP_QUALITY, s, 4.0 * (ne + 1) + 8.0 * 6.0 * m.counts[3] + 8.0 * ne +
      16.0 * m.counts[3] + 24.0 * m.counts[0] + 8.0 * m.counts[3] + 4.0 * ne + 16.0 * ne);
  u32 const qb = std::min<u32>(tuned(TK_QUALITY_BLOCK), 128u);
  CK(launch_kernel(k_swap_quality, dim3(grid_for(ne, qb)), dim3(qb), 0, s, ne, te.offs, te.adj, te.dirs, m.ask_down(1, 0),
      m.ask_down(3, 0), m.coords(), eq, m.fp32_filter ? fp32_stats_dev() : nullptr, sel.cand,
      sel.quals, sel.rs, sel.codes, any));
  CK_LAUNCH();
  if (!deferred && !read_u32(any, s)) return false;
  sel.ind = find_indset(m, 1, sel.cand, sel.quals, !deferred);
  return true;
}

// swap_interior + swap_ents (swap.cpp:27-97)
// deferred: the selection's flag and the set's outcome come back with the
// counts; with no swap kept it frees what it made and returns false
static bool swap_build(Mesh& m, SwapSel const& sel, bool deferred)
{
  cudaStream_t s = m.s;
  u32 ne = m.count(1), nv = m.count(0), dim = m.dim;
  Mesh* out = m.spawn();
  out->set_ents(0, nv, nullptr);
  for (auto const& t : m.tags[0]) {
    size_t bytes = (size_t)nv * t.ncomps * tag_esz(t.type);
    void* d = dev_alloc(bytes, s);
    CK(cudaMemcpyAsync(d, t.data, bytes, cudaMemcpyDeviceToDevice, s));
    out->add_tag(0, t.type, t.name.c_str(), t.ncomps, t.transfer, d);
  }
  if (m.seg) {
    out->seg = dalloc<u32>(nv, s);
    CK(cudaMemcpyAsync(out->seg, m.seg, sizeof(u32) * nv, cudaMemcpyDeviceToDevice, s));
  }
  if (m.parallel && m.globals[0]) {
    u64* g = dalloc<u64>(nv, s);
    CK(cudaMemcpyAsync(g, m.globals[0], sizeof(u64) * nv, cudaMemcpyDeviceToDevice, s));
    out->set_globals(0, g);
  } else if (m.parallel && m.globals_iota[0]) {
    out->set_iota_globals(0);
  }
  UpAdj const& te = m.ask_up(1, 3);
  u32 const* voe1 = m.ask_down(1, 0);
  u32 const* vot = m.ask_down(3, 0);
  u32* same_of[4] = {nullptr, nullptr, nullptr, nullptr};
  u32 nsame_of[4] = {0, 0, 0, 0};
  // the products and survivors of every dimension are counted first, their
  // totals landing in mailbox slots 20 + 2 (ed - 1) and 21 + 2 (ed - 1), so
  // one read-back serves all dimensions
  u32 const ed0 = m.full ? 1u : dim;
  u32* gen_offs_of[4] = {nullptr, nullptr, nullptr, nullptr};
  // each kept entity's new id, written by the survivors' scan for the
  // dimensions whose upward adjacency is carried
  u32* newid_of[4] = {nullptr, nullptr, nullptr, nullptr};
  // every dimension's two scans run together in one launch
  ScanJob sj[6];
  u32 nsj = 0;
  u32* scan_in[6] = {};
  for (u32 ed = ed0; ed <= dim; ++ed) {
    u32 n = m.count(ed);
    u32* cnt = dalloc<u32>(ne, s);
    CK(launch_kernel(k_swap_counts, dim3(grid_for(ne)), dim3(BLOCK), 0, s, ne, ed, sel.ind,
        sel.rs, cnt));
    CK_LAUNCH();
    gen_offs_of[ed] = dalloc<u32>((size_t)ne + 1, s);
    scan_in[nsj] = cnt;
    sj[nsj++] = ScanJob{cnt, gen_offs_of[ed], m.mb->dev + 20 + 2 * (ed - 1), nullptr, ne, 0};
    u32* same = dalloc<u32>(n, s);
    if (n) {
      u32 const lph = deg(ed, 1);
      auto k = lph == 1 ? k_swap_same<1> : lph == 3 ? k_swap_same<3> : k_swap_same<6>;
      CK(launch_kernel(k, dim3(grid_for(n)), dim3(BLOCK), 0, s, n,
          ed == 1 ? nullptr : m.ask_down(ed, 1), sel.ind, same));
      CK_LAUNCH();
    }
    if (carried_high(m, ed)) newid_of[ed] = dalloc<u32>(n ? n : 1, s);
    same_of[ed] = dalloc<u32>((size_t)n + 1, s);
    scan_in[nsj] = same;
    sj[nsj++] = ScanJob{same, same_of[ed], m.mb->dev + 21 + 2 * (ed - 1), newid_of[ed], n, 0};
  }
  exscan_jobs(sj, nsj, s);
  for (u32 k = 0; k < nsj; ++k) dev_free(scan_in[k], s);
  m.mb->fetch(s, deferred ? INDSET_FETCH_SLOTS : 26);
  if (deferred) {
    auto abandon = [&] {
      delete out;
      for (u32 d = 0; d < 4; ++d) {
        dev_free(same_of[d], s);
        dev_free(gen_offs_of[d], s);
        dev_free(newid_of[d], s);
      }
    };
    try {
      indset_check(m);
    } catch (...) {
      abandon();
      throw;
    }
    if (!m.mb->host[6]) {  // no swap kept: the set is empty
      abandon();
      last_pass_stats().indset_rounds = 0;
      return false;
    }
  }
  for (u32 ed = ed0; ed <= dim; ++ed) {
    u32 n = m.count(ed), vpe = deg(ed, 0);
    u32 ngen = m.mb->host[20 + 2 * (ed - 1)], nsame = m.mb->host[21 + 2 * (ed - 1)];
    u32* gen_offs = gen_offs_of[ed];
    u32* same_offs = same_of[ed];
    u32* conn = dalloc<u32>((size_t)(nsame + ngen) * vpe, s);
    expand_scaled(m.ask_down(ed, 0), same_offs, 1, n, vpe, 4, conn, s);
    CK(launch_kernel(k_swap_cavity, dim3(ceil_div(ne, 128)), dim3(128), 0, s, ne, ed, sel.ind, sel.codes, gen_offs, te.offs,
        te.adj, te.dirs, voe1, vot, conn + (size_t)nsame * vpe));
    CK_LAUNCH();
    out->set_ents(ed, nsame + ngen, conn);
    if (m.full) {
      // setup_swap (inherit.cpp:159-175)
      Doms d;
      d.ndoms[0] = n;
      d.offs[0] = same_offs;
      d.ngen[0] = nsame;
      d.ndoms[1] = ne;
      d.offs[1] = gen_offs;
      d.ngen[1] = ngen;
      d.finish();
      inherit_class(m, *out, ed, d);
    }
    if (m.parallel) inherit_globals(*out, ed);
    if (ed == dim) {
      bool any_f64 = false;
      for (auto const& t : m.tags[ed])
        if (t.type == T_F64) any_f64 = true;
      if (any_f64) {
        double* sizes = out->element_sizes();
        for (auto const& t : m.tags[ed]) {
          if (t.type != T_F64 || t.transfer != X_CONSERVE) continue;
          u32 nc = t.ncomps;
          if (nc > MAX_NCOMPS) throw Failure(E_ARG, "conserved field wider than 32");
          double* data = dalloc<double>((size_t)(nsame + ngen) * nc, s);
          expand_scaled(t.data, same_offs, 1, n, nc, 8, data, s);
          CK(launch_kernel(k_swap_conserve, dim3(grid_for(ne)), dim3(BLOCK), 0, s, ne, nc, nsame, gen_offs, te.offs,
              te.adj, sizes, static_cast<double const*>(t.data), data + (size_t)nsame * nc));
          CK_LAUNCH();
          out->add_tag(ed, T_F64, t.name.c_str(), nc, t.transfer, data);
        }
        dev_free(sizes, s);
      }
      for (auto const& t : m.tags[ed]) {
        if (t.type != T_F64 || t.transfer != X_POINTWISE) continue;
        u32 nc = t.ncomps;
        double* data = dalloc<double>((size_t)(nsame + ngen) * nc, s);
        expand_scaled(t.data, same_offs, 1, n, nc, 8, data, s);
        CK(launch_kernel(k_swap_fit, dim3(grid_for(ne)), dim3(BLOCK), 0, s, ne, nc, gen_offs, te.offs, te.adj,
            static_cast<double const*>(t.data), data + (size_t)nsame * nc));
        CK_LAUNCH();
        out->add_tag(ed, T_F64, t.name.c_str(), nc, t.transfer, data);
      }
    }
    dev_free(gen_offs, s);
    nsame_of[ed] = nsame;
  }
  same_of[0] = dalloc<u32>((size_t)nv + 1, s);  // vertices all survive, in order
  iota_u32(same_of[0], nv + 1, 1, s);
  nsame_of[0] = nv;
  // downward adjacency of the survivors carries over; the products are searched
  carry_down_all(m, *out, same_of, nsame_of);
  carry_up_all(m, *out, same_of, nsame_of, newid_of);
  for (u32 h = 0; h <= dim; ++h) dev_free(newid_of[h], s);
  for (u32 d = 0; d < 4; ++d) dev_free(same_of[d], s);
  m.overwrite(out);
  return true;
}

u32 swap_slivers(Mesh& m, double gq, u32 nlayers)
{
  if (m.dim != 3) throw Failure(E_ARG, "swap_slivers needs a 3D mesh");
  PassStats& st = last_pass_stats();
  st = PassStats();
  st.op = 3;
  st.elems_in = m.count(3);
  SwapSel sel;
  bool ok = false;
  // the selection's flag and the set's outcome come back with the build's
  // first read-back: two host waits fewer per pass
  bool const deferred = true;
  try {
    ok = swap_select(m, gq, nlayers, sel, nullptr, nullptr, nullptr, deferred);
    if (ok) {
      seg_tally(m, 1, sel.ind);
      st.nselected = 0;
      ok = swap_build(m, sel, deferred);
      if (ok) st.elems_out = m.count(3);
    }
  } catch (...) {
    sel.free(m.s);
    throw;
  }
  sel.free(m.s);
  return ok ? 1 : 0;
}

u32 swap_sets(Mesh& m, double gq, u32 nlayers, u32* slivers, u32* cand, u32* interior,
    u32* good, double* quals, u32* ring_sizes, u32* indset)
{
  cudaStream_t s = m.s;
  if (m.dim != 3) throw Failure(E_ARG, "swap_slivers needs a 3D mesh");
  u32 ne = m.count(1);
  CK(cudaMemsetAsync(good, 0, sizeof(u32) * ne, s));
  CK(cudaMemsetAsync(quals, 0, sizeof(double) * ne, s));
  CK(cudaMemsetAsync(ring_sizes, 0, sizeof(u32) * ne, s));
  CK(cudaMemsetAsync(indset, 0, sizeof(u32) * ne, s));
  SwapSel sel;
  bool ok = swap_select(m, gq, nlayers, sel, slivers, cand, interior);
  if (sel.quals) {
    CK(cudaMemcpyAsync(good, sel.cand, sizeof(u32) * ne, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(quals, sel.quals, sizeof(double) * ne, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ring_sizes, sel.rs, sizeof(u32) * ne, cudaMemcpyDeviceToDevice, s));
  }
  if (ok) CK(cudaMemcpyAsync(indset, sel.ind, sizeof(u32) * ne, cudaMemcpyDeviceToDevice, s));
  stream_sync(s);
  sel.free(s);
  return ok ? 1 : 0;
}

}  // namespace osh
