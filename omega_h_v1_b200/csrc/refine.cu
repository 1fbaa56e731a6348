// Edge refinement on sm_100a: refine_by_size / uniformly_refine
// (refine.cpp:11-35, refine_common.cpp:29-190, refine_qualities.cpp:16-82,
// splits_to_domains.cpp:13-56, refine_topology.cpp:26-120,
// refine_nodal.cpp:10-46, refine_conserve.cpp, refine_fit.cpp).
//
// Numbering of the new mesh follows the reference exactly: entities that do
// not split keep their order; products follow, grouped by the dimension of
// the domain that produced them and ordered by that domain's index (exclusive
// scans of the split marks), with new vertices appended in split-edge order.
#include "passes.hpp"

namespace osh {

// refine_candidate (refine.cpp:11-15) fused with measure_edge (size.cpp:57)
// (optional) list, nlist: the candidates appended, a warp's in one counter
// update (nlist zero on entry); zero_q: every edge's goodness zeroed for
// the quality kernel, which then writes only the listed edges'
__global__ void k_refine_candidates(u32 ne, u32 const* __restrict__ voe,
    double const* __restrict__ x, double const* __restrict__ h, SegView sv,
    Fp32Stats* fs, u32* __restrict__ cand, u32* any, u32* zero2, u32* __restrict__ list,
    u32* nlist, double* __restrict__ zero_q)
{
  pdl_wait();
  // (optional) two flags the quality kernel that follows sets, zeroed here
  // instead of by a memset of their own
  if (zero2 && blockIdx.x == 0 && threadIdx.x < 2) zero2[threadIdx.x] = 0;
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  u32 c = 0;
  bool decided = false, rechecked = false, flipped = false;
  if (i < ne) {
    u32 a = voe[i * 2], b = voe[i * 2 + 1];
    double xa[3], xb[3];
    load3(x, a, xa);
    load3(x, b, xb);
    int r32 = fs ? edge_ratio_side_f32(xa, xb, h[a], h[b], 1.0) : 0;
    if (r32) {
      decided = true;
      c = r32 > 0;
    }
    if (!r32 || fs->audit) {
      rechecked = !r32;
      double len = sqrt(sqdist3(xb, xa));
      double want = (h[a] + h[b]) / 2;
      u32 c64 = (len / want) > 1.0;
      flipped = r32 && c64 != c;
      c = c64;
    }
    c = c && seg_acts(sv, a);
    cand[i] = c;
    if (zero_q) zero_q[i] = 0.0;
  }
  if (fs) fp32_count_warp(fs, decided, rechecked, decided && fs->audit, flipped);
  unsigned const want = __ballot_sync(0xffffffffu, c != 0);
  if (want && (threadIdx.x & 31) == 0) atomicOr(any, 1u);
  if (list && want) {
    u32 const lane = threadIdx.x & 31, leader = __ffs(want) - 1;
    u32 base = 0;
    if (lane == leader) base = atomicAdd(nlist, (u32)__popc(want));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (c) list[base + __popc(want & ((1u << lane) - 1u))] = i;
  }
}

// the two children of element e (split at its edge of direction dir)
// around the midpoint `split`, in the reference's order
__device__ inline void refine_child(u32 dim, u32 const* __restrict__ ve, u32 dir, u32 k,
    double const* __restrict__ x, double const* split, double (*ex)[3])
{
  u32 vpe = deg(dim, 0);
  u32 o = canon(dim, 1, 0, dir, k);
  u32 base = opp(dim, 0, o);
  for (u32 l = 0; l + 1 < vpe; ++l) load3(x, ve[canon(dim, dim - 1, 0, base, l)], ex[l]);
  ex[vpe - 1][0] = split[0];
  ex[vpe - 1][1] = split[1];
  ex[vpe - 1][2] = split[2];
}

// refine_quality (refine_qualities.cpp:16-82) for edges, require_better = 0:
// the worst child of every element around the edge, split at its midpoint.
// With the filter: the children's estimates first; the edge is rejected on
// them when every child is surely upright and the worst surely below the
// floor; otherwise only the children whose lower bound reaches the lowest
// upper bound seen (they alone can hold the minimum) are computed in double.
// (Measured alternatives, both slower over an adapt: a group of 8 lanes per
// candidate edge, each lane some of its children, at 105 registers against
// 82; and one wave of resident blocks striding over the edges, which left
// the passes with many candidates to the threads that drew the most.)
//
// With a list (the candidate kernel's, nlist of them): a grid of the blocks
// that fit at once strides over the listed edges in block-wide steps (the
// candidates in order, so each thread draws as many as any other), and the
// goodness of the other edges was zeroed before. Without one: a thread per
// edge, its candidacy read from cand.
template <u32 DIM>
__global__ void k_refine_quality(u32 ne, u32 const* __restrict__ list,
    u32 const* __restrict__ nlist, u32 const* __restrict__ voe1,
    u32 const* __restrict__ voe, u32 const* __restrict__ eo_offs,
    u32 const* __restrict__ eo, u32 const* __restrict__ eo_dirs,
    double const* __restrict__ x, double qual_floor, SegView sv, Fp32Stats* fs,
    u32* __restrict__ cand, double* __restrict__ out, u32* any, u32* inverted)
{
  pdl_wait();
  constexpr u32 dim = DIM;  // the element dimension (2 or 3): loops over
                            // an element's vertices unroll, corners stay in registers
  u32 const n = list ? *nlist : ne;
  for (u32 base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    u32 const t = base + threadIdx.x;
    u32 const i = t < n ? (list ? list[t] : t) : 0u;
    u32 keep = 0;
    bool decided = false, rechecked = false, audited = false, flipped = false;
    if (t < n && (list || cand[i])) {
      constexpr u32 vpe = deg(dim, 0);
      double const perfect = dim == 3 ? perfect_tet_quality() : perfect_tri_quality();
      u32 a = voe1[i * 2], b = voe1[i * 2 + 1];
      double split[3];
      // average_element_field: (0 + x_a + x_b) / 2 per component
      for (u32 c = 0; c < 3; ++c) {
        double acc = 0;
        acc += x[a * 3 + c];
        acc += x[b * 3 + c];
        split[c] = acc / 2u;
      }
      double const fl = seg_floor(sv, a, qual_floor);
      u32 const f = eo_offs[i], e = eo_offs[i + 1];
      // filtered: 0 = no decision on estimates, 1 = rejected on them,
      // 2 = minimum over the children that can hold it
      int filtered = 0;
      double minq = 1;
      if (fs && dim == 3) {
        float const k6 = tet_k6_f32();
        float upper = 1.0f;
        bool upright = true;
        unsigned long long need = 0;  // children (2 per element) that can hold the minimum
        bool all = 2 * (e - f) > 64;
        for (u32 j = f; j < e; ++j) {
          u32 const* ve = voe + (size_t)eo[j] * vpe;
          for (u32 k = 0; k < 2; ++k) {
            double ex[4][3];
            refine_child(dim, ve, eo_dirs[j], k, x, split, ex);
            Q32 q = tet_quality_f32(ex, k6);
            float lo = q32_lo(q);
            upright = upright && lo > 0.0f;
            upper = fminf(upper, q32_hi(q));
            if (lo <= upper && !all) need |= 1ull << (2 * (j - f) + k);
          }
        }
        if (upright && (double)upper < fl) {
          filtered = 1;
          decided = true;
        } else if (upright) {
          filtered = 2;
          rechecked = true;
          for (u32 j = f; j < e; ++j) {
            u32 const* ve = voe + (size_t)eo[j] * vpe;
            for (u32 k = 0; k < 2; ++k) {
              if (!all && !((need >> (2 * (j - f) + k)) & 1ull)) continue;
              double ex[4][3];
              refine_child(dim, ve, eo_dirs[j], k, x, split, ex);
              double q = tet_quality(ex, perfect);
              if (fs->audit) fp32_note_error(fs, tet_quality_f32(ex, k6), q);
              if (q < minq) minq = q;
            }
          }
        }
        if (filtered && fs->audit) {
          // the double path's result, every child in order, and every
          // estimate against its double value
          audited = true;
          double m64 = 1;
          for (u32 j = f; j < e; ++j) {
            u32 const* ve = voe + (size_t)eo[j] * vpe;
            for (u32 k = 0; k < 2; ++k) {
              double ex[4][3];
              refine_child(dim, ve, eo_dirs[j], k, x, split, ex);
              double q = tet_quality(ex, perfect);
              fp32_note_error(fs, tet_quality_f32(ex, k6), q);
              if (q < m64) m64 = q;
            }
          }
          bool keep64 = !(m64 < fl);
          flipped = filtered == 1 ? keep64
                                  : (keep64 != !(minq < fl) || (keep64 && m64 != minq));
        }
      }
      if (!filtered) {
        for (u32 j = f; j < e; ++j) {
          u32 const* ve = voe + (size_t)eo[j] * vpe;
          for (u32 k = 0; k < 2; ++k) {
            double ex[4][3];
            refine_child(dim, ve, eo_dirs[j], k, x, split, ex);
            double q = dim == 3 ? tet_quality(ex, perfect) : tri_quality(ex, 0, perfect);
            if (!(q > 0)) atomicOr(inverted, 1u);
            if (q < minq) minq = q;
          }
        }
      }
      if (filtered == 1 || minq < fl) {
        cand[i] = 0;
      } else {
        out[i] = minq;
        keep = 1;
      }
    }
    // every edge's goodness is written here (with a list: the listed ones)
    if (t < n && !keep) out[i] = 0.0;
    if (fs && dim == 3) fp32_count_warp(fs, decided, rechecked, audited, flipped);
    if (__any_sync(0xffffffffu, keep) && (threadIdx.x & 31) == 0) atomicOr(any, 1u);
  }
}

// refine_node (refine_nodal.cpp:10-25)
// every double vertex field of the refined mesh in one launch (blockIdx.y:
// the field): the old vertices' values copied, then each new vertex's the
// average of its edge's two vertices
constexpr u32 MAX_NODAL_FIELDS = 8;
struct NodalFields {
  double const* f[MAX_NODAL_FIELDS];
  double* out[MAX_NODAL_FIELDS];
  u32 nc[MAX_NODAL_FIELDS];
};

// (split: the split edges in order, nsplit of them; the k-th one's new
// vertex is nv + k)
__global__ void k_refine_nodal(u32 nsplit, u32 nv, u32 const* __restrict__ voe,
    u32 const* __restrict__ split, const __grid_constant__ NodalFields fields)
{
  pdl_wait();
  u32 const nc = fields.nc[blockIdx.y];
  double const* __restrict__ f = fields.f[blockIdx.y];
  double* __restrict__ out = fields.out[blockIdx.y];
  u64 const ncopy = (u64)nv * nc, total = ncopy + nsplit;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (u64)gridDim.x * blockDim.x) {
    if (t < ncopy) {
      out[t] = f[t];
      continue;
    }
    u32 const k = (u32)(t - ncopy), i = split[k];
    u32 a = voe[i * 2], b = voe[i * 2 + 1];
    double* o = out + (size_t)(nv + k) * nc;
    for (u32 c = 0; c < nc; ++c) {
      double acc = 0;
      acc += f[(size_t)a * nc + c];
      acc += f[(size_t)b * nc + c];
      o[c] = acc / 2u;
    }
  }
}

// segment of each new vertex: the segment of its edge's first vertex
__global__ void k_refine_seg(u32 ne, u32 nv, u32 const* __restrict__ voe,
    u32 const* __restrict__ gen_offs, u32 const* __restrict__ seg, u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne || gen_offs[i] == gen_offs[i + 1]) return;
  out[nv + gen_offs[i]] = seg[voe[i * 2]];
}

// split_to_domain (splits_to_domains.cpp:13-31): whether a domain holds a
// split edge (SPD edges per domain entity, a compile-time count: the loads
// of all of them are issued before any is used). Which edge (the first in
// local order) and its new vertex are found again by the topology kernel
// for the split domains alone.
template <u32 SPD>
__device__ inline bool first_split_edge(u32 const* __restrict__ sod,
    u32 const* __restrict__ gen_offs, u32 i, u32& dir, u32& vert_off)
{
  u32 sv[SPD], a[SPD], b[SPD];
#pragma unroll
  for (u32 j = 0; j < SPD; ++j) sv[j] = sod[(size_t)i * SPD + j];
#pragma unroll
  for (u32 j = 0; j < SPD; ++j) {
    a[j] = gen_offs[sv[j]];
    b[j] = gen_offs[sv[j] + 1];
  }
  bool w = false;
#pragma unroll
  for (u32 j = SPD; j-- > 0;)
    if (a[j] != b[j]) {  // the first split edge in local order wins
      w = true;
      dir = j;
      vert_off = a[j];
    }
  return w;
}

// (optional) the vertices' maps on the threads past the domains: their
// domain offsets (no vertex splits: zeros) and their identity survivor maps
struct VertexMaps {
  u32 nv;
  u32* zero;
  u32* same;
  u32* newid;
};

__device__ inline void vertex_maps(VertexMaps const& vm, u32 i)
{
  if (i > vm.nv) return;
  vm.zero[i] = 0;
  vm.same[i] = i;
  if (vm.newid && i < vm.nv) vm.newid[i] = i;
}

// The same marks from the split edges' side: the faces and elements in the
// upward rows of each split edge, stamped with a generation in kept marks
// (no array of every domain entity is written or read here). A thread per
// split edge of the list, whose length is the split edges' scan total,
// read here; a capped grid strides over the list, then over the vertices'
// maps.
struct SplitMark {
  u32 const* offs;  // up(1, dd) of the mesh being refined
  u32 const* adj;
  u32* marks;
  u32 gen;
};
struct SplitMarks {
  SplitMark d[2];  // domain dimensions 2 and 3 (marks null: not this way)
};

__global__ void k_mark_split_domains(u32 const* __restrict__ list,
    u32 const* __restrict__ nsplit_at, SplitMarks sm, VertexMaps vm)
{
  pdl_wait();
  u32 const stride = gridDim.x * blockDim.x, t0 = blockIdx.x * blockDim.x + threadIdx.x;
  u32 const nsplit = *nsplit_at;
  for (u32 t = t0; t < nsplit; t += stride) {
    u32 const e = list[t];
#pragma unroll
    for (u32 q = 0; q < 2; ++q) {
      SplitMark const& d = sm.d[q];
      if (!d.marks) continue;
      for (u32 j = d.offs[e], f = d.offs[e + 1]; j < f; ++j) d.marks[d.adj[j]] = d.gen;
    }
  }
  if (vm.zero)
    for (u32 t = t0; t <= vm.nv; t += stride) vertex_maps(vm, t);
}

template <u32 SPD>
__global__ void k_split_to_domain(u32 nd, u32 const* __restrict__ sod,
    u32 const* __restrict__ gen_offs, u32* __restrict__ will, VertexMaps vm)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nd) {
    if (vm.zero) vertex_maps(vm, i - nd);
    return;
  }
  u32 d, v;
  will[i] = first_split_edge<SPD>(sod, gen_offs, i, d, v) ? 1u : 0u;
}

// refine_domain_entity (refine_topology.cpp:26-64), for every product and
// domain dimension of a pass in one launch (blockIdx.y: the pair's job), a
// thread per split domain entity from the list of them in order. The domain's split edge and the new vertex on it: the edge
// itself for edge domains, else its first split edge (sod: the domain's
// edges).
struct TopoJob {
  u32 prod, dd, nsplit;
  u32 const* list;
  u32 const* vod;
  u32 const* sod;
  u32* out;
};
struct TopoJobs {
  TopoJob j[6];  // every (product, domain) dimension pair of a 3D pass
};

__global__ void k_refine_topology(const __grid_constant__ TopoJobs jobs,
    u32 const* __restrict__ gen_offs, u32 nv)
{
  pdl_wait();
  TopoJob const jb = jobs.j[blockIdx.y];
  u32 const dd = jb.dd, prod = jb.prod;
  u32 t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= jb.nsplit) return;
  u32 const i = jb.list[t];
  u32 di = 0, voff = 0;
  if (dd == 1)
    voff = gen_offs[i];
  else if (dd == 2)
    first_split_edge<3>(jb.sod, gen_offs, i, di, voff);
  else
    first_split_edge<6>(jb.sod, gen_offs, i, di, voff);
  u32 base_dim = prod - 1, opp_dim = dd - 1 - base_dim;
  u32 ops = deg(1, opp_dim), vpp = deg(prod, 0), vpb = vpp - 1, vpd = deg(dd, 0);
  // the t-th split domain's products are the t-th group (its offset is t)
  u32* p = jb.out + (size_t)t * ops * vpp;
  for (u32 j = 0; j < ops; ++j) {
    u32 o = canon(dd, 1, opp_dim, di, j);
    u32 b = opp(dd, opp_dim, o);
    for (u32 k = 0; k < vpb; ++k) p[k] = jb.vod[(size_t)i * vpd + canon(dd, base_dim, 0, b, k)];
    p[vpb] = nv + voff;
    p += vpp;
  }
}

// refine_conserve_elem / refine_fit_elem (refine_conserve.cpp:10-21,
// refine_fit.cpp:10-20): each product gets the value (divided by the number
// of products when conserving)
__global__ void k_refine_elem_field(u32 n, u32 const* __restrict__ offs, u32 k,
    u32 nc, int conserve, double const* __restrict__ in, double* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 f = offs[i] * k, e = offs[i + 1] * k;
  double denom = e - f;
  for (u32 j = f; j < e; ++j)
    for (u32 c = 0; c < nc; ++c)
      out[(size_t)j * nc + c] = conserve ? in[(size_t)i * nc + c] / denom : in[(size_t)i * nc + c];
}

static u32 prods_per_dom(u32 dom, u32 src, u32 prod)
{
  // get_prods_per_dom (refine_topology.cpp:110-120)
  if (prod == 0) return dom == src ? 1 : 0;
  u32 base = prod - 1, o = dom - 1 - base;
  if (src < o) return 0;
  return deg(src, o);
}

struct Splits {
  u32* offs = nullptr;
  u32* list = nullptr;  // the split entities, in order (nsplit of them)
  u32 nsplit = 0;
};

// the split edges' scan: each edge's new-vertex offset (gen_offs), the split
// edges in order (list), and the surviving edges' maps (same, and newid when
// the edges' upward adjacency is carried) -- everything the edges need as a
// domain, from the one scan (refine_build takes list, same and newid over)
struct EdgeSplits {
  u32* gen_offs = nullptr;
  u32* list = nullptr;
  u32* same = nullptr;
  u32* newid = nullptr;
};

// the vertices' maps alone (a pass without triangle or tet domains)
__global__ void k_vertex_maps(VertexMaps vm)
{
  pdl_wait();
  vertex_maps(vm, blockIdx.x * blockDim.x + threadIdx.x);
}

// returns the number of split edges (read back with the domain counts).
// deferred: the independent set's outcome comes back with the same
// read-back; nothing to split (or a failed set) leaves the mesh unchanged.
static u32 refine_build(Mesh& m, EdgeSplits const& es, bool deferred, bool uniform)
{
  u32 const* gen_offs = es.gen_offs;
  cudaStream_t s = m.s;
  u32 dim = m.dim, src = 1;
  u32 nv = m.count(0), ns = m.count(src);
  Mesh* out = m.spawn();
  // splits_to_domains for every domain dimension; the edges' count is the
  // number of split edges, so one read-back sizes everything below
  Splits sp[4];
  // products of every dimension (refine_common.cpp:90-123, inherit.cpp:104-138):
  // the survivors of each (same_of) and, for the dimensions whose upward
  // adjacency is carried, each kept entity's new id (newid_of). A domain
  // splits (mark 1) or survives (mark 0), so the domains' scan writes both
  // as the scan of the complement; vertices all survive (identity maps).
  u32* same_of[4] = {nullptr, nullptr, nullptr, nullptr};
  u32 nsame_of[4] = {0, 0, 0, 0};
  u32* newid_of[4] = {nullptr, nullptr, nullptr, nullptr};
  auto is_prod = [&](u32 prod) { return m.full || prod == 0 || prod == dim; };
  u32* zero_v = dalloc<u32>((size_t)nv + 1, s);
  same_of[0] = dalloc<u32>((size_t)nv + 1, s);
  if (carried_high(m, 0)) newid_of[0] = dalloc<u32>(nv ? nv : 1, s);
  // written by the first split-mark launch below (or on their own)
  VertexMaps vm{nv, zero_v, same_of[0], newid_of[0]};
  sp[0].offs = zero_v;
  // the edges as domains: the split edges' scan (the caller owns gen_offs)
  sp[1].offs = es.gen_offs;
  sp[1].list = es.list;
  same_of[1] = es.same;
  newid_of[1] = es.newid;
  u32* will[4] = {nullptr, nullptr, nullptr, nullptr};
  ScanJob jobs[4];
  u32 njobs = 0;
  // A domain dimension whose upward rows from the edges the mesh holds is
  // marked from the split edges (k_mark_split_domains) unless every edge
  // splits; the others by a pass over every domain entity
  SplitMarks sm{};
  bool any_sparse = false;
  for (u32 dd = 2; dd <= dim; ++dd) {
    if (!m.has_dim(dd)) continue;
    u32 nd = m.count(dd);
    if (!uniform && nd && m.have_up[1][dd]) {
      SplitMark& d = sm.d[dd - 2];
      d.offs = m.up[1][dd].offs;
      d.adj = m.up[1][dd].adj;
      d.marks = stream_marks(KEPT_SPLIT + dd, nd, s, &d.gen);
      any_sparse = true;
      sp[dd].offs = dalloc<u32>((size_t)nd + 1, s);
      sp[dd].list = dalloc<u32>(nd, s);
      ScanJob j{d.marks, sp[dd].offs, m.mb->dev + 8 + dd, nullptr, nd, 2, sp[dd].list};
      j.stamp = d.gen;
      if (is_prod(dd)) {
        same_of[dd] = j.comp = dalloc<u32>((size_t)nd + 1, s);
        if (carried_high(m, dd)) newid_of[dd] = j.comp_newid = dalloc<u32>(nd, s);
      }
      jobs[njobs++] = j;
      continue;
    }
    u32 const* sod = m.ask_down(dd, 1);
    will[dd] = dalloc<u32>(nd, s);
    if (nd || vm.zero) {
      u64 const nthreads = (u64)nd + (vm.zero ? (u64)nv + 1 : 0);
      auto k = dd == 2 ? k_split_to_domain<3> : k_split_to_domain<6>;
      CK(launch_kernel(k, dim3(grid_for(nthreads)), dim3(BLOCK), 0, s, nd, sod, gen_offs,
          will[dd], vm));
      CK_LAUNCH();
      vm.zero = nullptr;  // done
    }
    sp[dd].offs = dalloc<u32>((size_t)nd + 1, s);
    sp[dd].list = dalloc<u32>(nd ? nd : 1, s);
    ScanJob j{will[dd], sp[dd].offs, m.mb->dev + 8 + dd, nullptr, nd, 0, sp[dd].list};
    if (is_prod(dd)) {
      same_of[dd] = j.comp = dalloc<u32>((size_t)nd + 1, s);
      if (carried_high(m, dd)) newid_of[dd] = j.comp_newid = dalloc<u32>(nd ? nd : 1, s);
    }
    jobs[njobs++] = j;
  }
  if (any_sparse) {
    // the split edges' count is their scan's total, gen_offs[n_edges]
    u32 const grid = std::min<u32>(grid_for((u64)std::max(ns, nv) + 1), 148u * 8u);
    CK(launch_kernel(k_mark_split_domains, dim3(grid), dim3(BLOCK), 0, s, es.list,
        gen_offs + ns, sm, vm));
    CK_LAUNCH();
    vm.zero = nullptr;  // done
  }
  if (vm.zero) {
    CK(launch_kernel(k_vertex_maps, dim3(grid_for((u64)nv + 1)), dim3(BLOCK), 0, s, vm));
    CK_LAUNCH();
  }
  // the other domains' scans in one launch
  exscan_jobs(jobs, njobs, s);
  for (u32 dd = 1; dd <= dim; ++dd) dev_free(will[dd], s);
  m.mb->fetch(s, deferred ? INDSET_FETCH_SLOTS : 16);
  if (deferred) {
    auto abandon = [&] {
      delete out;
      for (u32 dd = 0; dd <= dim; ++dd) {
        if (dd != 1) dev_free(sp[dd].offs, s);
        dev_free(sp[dd].list, s);
        dev_free(same_of[dd], s);
        dev_free(newid_of[dd], s);
      }
    };
    try {
      indset_check(m);
    } catch (...) {
      abandon();
      throw;
    }
    if (!m.mb->host[1]) {  // no good candidate: the set is empty
      abandon();
      last_pass_stats().indset_rounds = 0;
      // choose_refinement_indset exchanges the edge qualities of a parallel
      // mesh once any edge is a candidate
      if (m.parallel && !m.seg && (uniform || m.mb->host[3])) m.note_exchange(1);
      return 0;
    }
  }
  for (u32 dd = 1; dd <= dim; ++dd)
    if (m.has_dim(dd)) sp[dd].nsplit = m.mb->host[8 + dd];
  u32 nsplit = sp[1].nsplit;
  // refine_verts (refine_common.cpp:29-54)
  u32 nv_out = nv + nsplit;
  out->set_ents(0, nv_out, nullptr);
  u32 const* voe1 = m.ask_down(1, 0);
  {
    NodalFields nf;
    u32 nfields = 0;
    u64 most = 0;
    auto flush = [&] {
      if (!nfields) return;
      u32 const gb = tuned(TK_GATHER_BLOCK);
      u32 gx = (u32)std::min<u64>(ceil_div(most, (u64)gb), 148u * 8u * 256u / gb);
      CK(launch_kernel(k_refine_nodal, dim3(gx ? gx : 1, nfields), dim3(gb), 0, s, nsplit, nv,
          voe1, es.list, nf));
      CK_LAUNCH();
      nfields = 0;
      most = 0;
    };
    for (auto const& t : m.tags[0]) {
      if (t.type != T_F64) continue;
      double* d = dalloc<double>((size_t)nv_out * t.ncomps, s);
      nf.f[nfields] = static_cast<double const*>(t.data);
      nf.out[nfields] = d;
      nf.nc[nfields] = t.ncomps;
      most = std::max<u64>(most, (u64)nv * t.ncomps + nsplit);
      if (++nfields == MAX_NODAL_FIELDS) flush();
      out->add_tag(0, T_F64, t.name.c_str(), t.ncomps, X_NOT, d);
    }
    flush();
  }
  if (m.parallel) inherit_globals(*out, 0);
  if (m.seg) {
    out->seg = dalloc<u32>(nv_out, s);
    CK(cudaMemcpyAsync(out->seg, m.seg, sizeof(u32) * nv, cudaMemcpyDeviceToDevice, s));
    if (ns) {
      CK(launch_kernel(k_refine_seg, dim3(grid_for(ns)), dim3(BLOCK), 0, s, ns, nv, voe1, gen_offs, m.seg, out->seg));
      CK_LAUNCH();
    }
  }
  TopoJobs tj;
  u32 ntj = 0, tmost = 0;
  double tbytes = 0;
  // the survivors' connectivity and every dimension's label copies, launched
  // together after the loop (8 jobs to a launch)
  std::vector<ExpandJob> copies;
  for (u32 prod = 0; prod <= dim; ++prod) {
    if (!m.full && 0 < prod && prod < dim) continue;
    u32 np = m.count(prod);
    Doms d;
    u32* same = same_of[prod];
    std::vector<ExpandJob> conn_job;
    d.ndoms[0] = np;
    d.offs[0] = same;
    d.scale[0] = 1;
    u32 first, last;
    if (m.full) {
      first = src > prod ? src : prod;
      last = dim;
    } else {
      first = last = (prod == 0) ? src : dim;
    }
    for (u32 dd = first; dd <= last; ++dd) {
      d.ndoms[dd] = m.count(dd);
      d.offs[dd] = sp[dd].offs;
      d.scale[dd] = prods_per_dom(dd, src, prod);
      d.ngen[dd] = sp[dd].nsplit * d.scale[dd];
      d.list[dd] = sp[dd].list;
      d.nlist[dd] = sp[dd].nsplit;
    }
    d.ngen[0] = np - sp[prod].nsplit;
    d.finish();
    if (prod) {
      u32 vpp = deg(prod, 0), nout = d.ngo[4];
      u32* conn = dalloc<u32>((size_t)nout * vpp, s);
      // the survivors' connectivity is copied with the class labels' copies
      ExpandJob cj;
      cj.in = m.ask_down(prod, 0);
      cj.offs = same;
      cj.out = conn;
      cj.k = 1;
      cj.n = np;
      cj.width = vpp;
      cj.esz = 4;
      conn_job.push_back(cj);
      // the products' vertices: one launch for every dimension, after
      // this loop (they write past the survivors' rows of each array)
      for (u32 dd = first; dd <= last; ++dd) {
        if (!d.ndoms[dd] || !d.scale[dd] || !sp[dd].nsplit) continue;
        u32 nd = sp[dd].nsplit;
        tj.j[ntj++] = TopoJob{prod, dd, nd, sp[dd].list, m.ask_down(dd, 0),
            dd == 1 ? nullptr : m.ask_down(dd, 1), conn + (size_t)d.ngo[dd] * vpp};
        tmost = std::max(tmost, nd);
        tbytes += 4.0 * nd + 4.0 * deg(dd, 0) * nd + 12.0 * deg(dd, 1) * nd +
            4.0 * vpp * (double)d.ngen[dd];
      }
      out->set_ents(prod, nout, conn);
      if (m.parallel) inherit_globals(*out, prod);
    }
    inherit_class(m, *out, prod, d, &conn_job, &copies);
    if (prod == dim) {
      for (int pass = 0; pass < 2; ++pass) {
        u32 want = pass == 0 ? X_CONSERVE : X_POINTWISE;
        for (auto const& t : m.tags[dim]) {
          if (t.type != T_F64 || t.transfer != want) continue;
          u32 nc = t.ncomps;
          double* data = dalloc<double>((size_t)d.ngo[4] * nc, s);
          expand_scaled(t.data, same, 1, np, nc, 8, data, s);
          if (d.ngen[dim]) {
            CK(launch_kernel(k_refine_elem_field, dim3(grid_for(np)), dim3(BLOCK), 0, s, np, sp[dim].offs,
                d.scale[dim], nc, pass == 0, static_cast<double const*>(t.data),
                data + (size_t)d.ngo[dim] * nc));
            CK_LAUNCH();
          }
          out->add_tag(dim, T_F64, t.name.c_str(), nc, t.transfer, data);
        }
      }
    }
    same_of[prod] = same;
    nsame_of[prod] = np - sp[prod].nsplit;
  }
  expand_many(copies, s);
  if (ntj) {
    PROBE(P_REFINE_TOPOLOGY, s, tbytes);
    CK(launch_kernel(k_refine_topology, dim3(grid_for(tmost), ntj), dim3(BLOCK), 0, s, tj,
        gen_offs, nv));
    CK_LAUNCH();
  }
  // downward adjacency of the survivors carries over; the products are searched
  carry_down_all(m, *out, same_of, nsame_of);
  carry_up_all(m, *out, same_of, nsame_of, newid_of);
  for (u32 h = 0; h <= dim; ++h) dev_free(newid_of[h], s);
  for (u32 dd = 0; dd <= dim; ++dd) {
    dev_free(same_of[dd], s);
    if (dd != 1) dev_free(sp[dd].offs, s);  // the edges' are the caller's gen_offs
    dev_free(sp[dd].list, s);
  }
  m.overwrite(out);
  return nsplit;
}

// choose_refinement_indset (refine_common.cpp:131-160) on a candidate array
// the caller owns; returns the independent set or nullptr when nothing
// qualifies. quals_out (optional) receives the goodness.
// uniform: every edge is a candidate; otherwise the candidate kernel of
// refine_by_size / refine_sets left "any candidate" in mailbox slot 3
// deferred (see refine_deferred): the set is returned unchecked, and the
// build's read-back brings its outcome and the flags
// zeroed: the candidate kernel already zeroed mailbox slots 1-2
// list, nlist (optional): the candidates listed by the candidate kernel,
// which also zeroed q_in (the goodness array this call then owns)
static u32* choose_refinement(Mesh& m, u32* cand, double qual_floor, double** quals_out,
    bool uniform, bool deferred = false, bool zeroed = false, u32 const* list = nullptr,
    u32 const* nlist = nullptr, double* q_in = nullptr)
{
  cudaStream_t s = m.s;
  u32 ne = m.count(1), dim = m.dim;
  double* q = q_in ? q_in : dalloc<double>(ne, s);
  if (dim < 2) CK(cudaMemsetAsync(q, 0, sizeof(double) * ne, s));
  u32* any = m.mb->dev + 1;
  u32* inverted = m.mb->dev + 2;
  if (!zeroed) CK(cudaMemsetAsync(any, 0, 2 * sizeof(u32), s));
  if (dim >= 2) {
    UpAdj const& eo = m.ask_up(1, dim, false);
    if (ne) {
      // refine_quality bytes (edges' up CSR, elements, coordinates, flags)
      double nel = m.counts[dim];
      PROBE(P_REFINE_QUALITY, s, 4.0 * (ne + 1) + 8.0 * deg(dim, 1) * nel + 8.0 * ne +
          4.0 * deg(dim, 0) * nel + 24.0 * m.counts[0] + 8.0 * ne + 8.0 * ne);
      u32 const qb = tuned(TK_QUALITY_BLOCK);
      auto kq = dim == 3 ? k_refine_quality<3> : k_refine_quality<2>;
      u32 grid = grid_for(ne, qb);
      if (list) {
        // the listed edges' goodness is written by the kernel, the rest is 0
        if (!q_in) CK(cudaMemsetAsync(q, 0, sizeof(double) * ne, s));
        grid = std::min(grid, resident_blocks(kq, qb));
      }
      CK(launch_kernel(kq, dim3(grid), dim3(qb), 0, s, ne, list, nlist, m.ask_down(1, 0),
          m.ask_down(dim, 0), eo.offs, eo.adj, eo.dirs, m.coords(), qual_floor, m.segview(),
          m.fp32_filter ? fp32_stats_dev() : nullptr, cand, q, any, inverted));
      CK_LAUNCH();
    }
  } else {
    m.mb->host[1] = max_u32(cand, ne, s) ? 1 : 0;
  }
  // The independent set runs without first reading back "any good
  // candidate": with none it settles in its first batch of rounds to the
  // empty set, and its first read-back brings the flags of mailbox slots
  // 1-3 with it (one host wait fewer per pass).
  u32* ind = ne ? find_indset(m, 1, cand, q, !deferred) : nullptr;
  if (deferred) {
    if (m.parallel && !m.seg) m.ensure_ghosting(1);
    dev_free(q, s);
    return ind;
  }
  if (!ne) m.mb->host[1] = m.mb->host[3] = 0;
  // choose_refinement_indset (refine_common.cpp:131-160) ghosts a parallel
  // mesh, and exchanges the edge qualities once any edge is a candidate
  if (m.parallel && !m.seg) {
    m.ensure_ghosting(1);
    bool any_cand = uniform ? ne > 0 : dim >= 2 ? m.mb->host[3] != 0 : m.mb->host[1] != 0;
    if (any_cand) m.note_exchange(1);
  }
  if (quals_out)
    *quals_out = q;
  else
    dev_free(q, s);
  if (!m.mb->host[1]) {
    dev_free(ind, s);
    last_pass_stats().indset_rounds = 0;
    return nullptr;
  }
  return ind;
}

// The independent set's outcome need not be read back on its own: it comes
// back with the build's first read-back, one host wait fewer per pass. (A
// parallel mesh's ghosting state that depends on the flags is set after
// that read-back: a pass that changes the mesh replaces that state anyway.)
static bool refine_deferred(Mesh& m)
{
  return m.count(1) && m.dim >= 2;
}

static u32 refine_common(Mesh& m, u32* cand, double qual_floor, bool uniform,
    bool zeroed = false, u32 const* list = nullptr, u32 const* nlist = nullptr,
    double* q_in = nullptr)
{
  cudaStream_t s = m.s;
  PassStats& st = last_pass_stats();
  st = PassStats();
  st.op = 1;
  st.elems_in = m.count(m.dim);
  u32 ne = m.count(1);
  bool const deferred = refine_deferred(m);
  u32* ind = choose_refinement(m, cand, qual_floor, nullptr, uniform, deferred, zeroed, list,
      nlist, q_in);
  if (!ind) return 0;
  seg_tally(m, 1, ind);
  // the split edges' scan, with their list and the surviving edges' maps
  // (the edges' count goes to mailbox slot 9 with the other domains')
  EdgeSplits es;
  es.gen_offs = dalloc<u32>((size_t)ne + 1, s);
  es.list = dalloc<u32>(ne ? ne : 1, s);
  if (m.full || m.dim == 1) {
    es.same = dalloc<u32>((size_t)ne + 1, s);
    if (carried_high(m, 1)) es.newid = dalloc<u32>(ne ? ne : 1, s);
  }
  {
    ScanJob j{ind, es.gen_offs, m.mb->dev + 9, nullptr, ne, 0, es.list};
    j.comp = es.same;
    j.comp_newid = es.newid;
    exscan_jobs(&j, 1, s);
  }
  dev_free(ind, s);
  u32 nsplit = 0;
  try {
    nsplit = refine_build(m, es, deferred, uniform);
  } catch (...) {
    dev_free(es.gen_offs, s);
    throw;
  }
  dev_free(es.gen_offs, s);
  if (!nsplit) return 0;  // a deferred set that came back empty
  st.nselected = nsplit;
  st.elems_out = m.count(m.dim);
  return 1;
}

u32 refine_by_size(Mesh& m, double qual_floor)
{
  cudaStream_t s = m.s;
  u32 ne = m.count(1);
  Tag* h = m.find_tag(0, "adapt_size");
  if (!h) throw Failure(E_ARG, "mesh has no adapt_size vertex field");
  u32* cand = dalloc<u32>(ne, s);
  u32* clist = dalloc<u32>(ne ? ne : 1, s);
  // the edges' goodness, zeroed by the candidate kernel; refine_common's
  // selection owns it from there
  double* q = m.dim >= 2 ? dalloc<double>(ne ? ne : 1, s) : nullptr;
  // mailbox slot 0: the candidates listed; slot 3: any candidate
  u32* nlist = m.mb->dev + 0;
  u32* any = m.mb->dev + 3;
  CK(cudaMemsetAsync(nlist, 0, 4 * sizeof(u32), s));  // slots 0-3
  if (ne) {
    PROBE(P_REFINE_CANDIDATES, s, 8.0 * ne + 32.0 * m.counts[0] + 4.0 * ne);
    CK(launch_kernel(k_refine_candidates, dim3(grid_for(ne)), dim3(BLOCK), 0, s, ne, m.ask_down(1, 0), m.coords(),
        static_cast<double const*>(h->data), m.segview(),
        m.fp32_filter ? fp32_stats_dev() : nullptr, cand, any, m.mb->dev + 1, clist, nlist, q));
    CK_LAUNCH();
  }
  // no separate check for "any candidate": with none, the quality kernel
  // keeps none and refine_common returns 0 after its single read-back
  u32 r = 0;
  try {
    r = refine_common(m, cand, qual_floor, false, ne != 0, clist, nlist, q);
  } catch (...) {
    dev_free(clist, s);
    dev_free(cand, s);
    throw;
  }
  dev_free(clist, s);
  dev_free(cand, s);
  return r;
}

void uniformly_refine(Mesh& m)
{
  u32 ne = m.count(1);
  u32* cand = dalloc<u32>(ne, m.s);
  fill_u32(cand, ne, 1, m.s);
  if (ne) refine_common(m, cand, 0.0, true);
  dev_free(cand, m.s);
}

u32 refine_sets(Mesh& m, double qual_floor, u32* cand_out, u32* good_out,
    double* quals_out, u32* indset_out)
{
  cudaStream_t s = m.s;
  u32 ne = m.count(1);
  Tag* h = m.find_tag(0, "adapt_size");
  if (!h) throw Failure(E_ARG, "mesh has no adapt_size vertex field");
  u32* any = m.mb->dev + 3;
  CK(cudaMemsetAsync(any, 0, sizeof(u32), s));
  CK(cudaMemsetAsync(indset_out, 0, sizeof(u32) * ne, s));
  if (ne) {
    CK(launch_kernel(k_refine_candidates, dim3(grid_for(ne)), dim3(BLOCK), 0, s, ne, m.ask_down(1, 0), m.coords(),
        static_cast<double const*>(h->data), m.segview(),
        m.fp32_filter ? fp32_stats_dev() : nullptr, cand_out, any, nullptr, nullptr, nullptr,
        nullptr));
    CK_LAUNCH();
  }
  CK(cudaMemcpyAsync(good_out, cand_out, sizeof(u32) * ne, cudaMemcpyDeviceToDevice, s));
  double* q = nullptr;
  u32* ind = choose_refinement(m, good_out, qual_floor, &q, false);
  CK(cudaMemcpyAsync(quals_out, q, sizeof(double) * ne, cudaMemcpyDeviceToDevice, s));
  dev_free(q, s);
  if (!ind) {
    stream_sync(s);
    return 0;
  }
  CK(cudaMemcpyAsync(indset_out, ind, sizeof(u32) * ne, cudaMemcpyDeviceToDevice, s));
  dev_free(ind, s);
  stream_sync(s);
  return 1;
}

}  // namespace osh
