// Batched adaptation of many meshes as one disjoint union (see batch.hpp).
//
// Concatenation: per dimension, the meshes' connectivity is laid end to end
// with each mesh's vertex ids shifted by the vertices before it, tags are
// laid end to end, and every vertex records its segment (mesh index). One
// launch per array does the copy for all meshes.
//
// Splitting: per dimension, a stable counting sort by segment (one warp per
// tile of entities builds a segment-major histogram of tiles, an exclusive
// scan turns it into positions, and the same warps scatter), then one launch
// per array writes every mesh's part straight into that mesh's own arrays,
// with vertex ids renumbered to the mesh's local numbering.
#include <algorithm>
#include <cfloat>
#include <chrono>

#include "batch.hpp"

namespace osh {

BatchStats& last_batch_stats()
{
  static thread_local BatchStats s;
  return s;
}

namespace {

constexpr u32 FULL_MASK = 0xffffffffu;
constexpr u32 SPLIT_TILE = 2048;   // entities per warp in the counting sort
constexpr u32 CAP_GRID = 148 * 16; // grid-stride kernels: 16 blocks per SM

u32 capped_grid(u64 n) { return n ? (u32)std::min<u64>(ceil_div(n, BLOCK), CAP_GRID) : 1; }

// index of the segment holding unit `unit`: offs[lo] <= unit < offs[lo + 1]
__device__ inline u32 find_seg(u32 nm, u32 const* __restrict__ offs, u32 unit)
{
  u32 lo = 0, hi = nm;
  while (hi - lo > 1) {
    u32 mid = (lo + hi) >> 1;
    if (offs[mid] <= unit)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// out[j] = src[m][j - offs[m]*width] (+ add[m]) for the segment m of unit j/width
template <class T>
__global__ void k_concat(u32 nm, T const* const* __restrict__ src, u32 const* __restrict__ offs,
    u32 width, T const* __restrict__ add, T* __restrict__ out)
{
  pdl_wait();
  u64 total = (u64)offs[nm] * width;
  for (u64 j = blockIdx.x * (u64)blockDim.x + threadIdx.x; j < total;
       j += (u64)gridDim.x * blockDim.x) {
    u32 m = find_seg(nm, offs, (u32)(j / width));
    T v = src[m][j - (u64)offs[m] * width];
    if (add) v += add[m];
    out[j] = v;
  }
}

// segment of every vertex of the union: the input's index, or, for an input
// that is itself a union, its own segment shifted by the segments before it
__global__ void k_seg_concat(u32 nm, u32 const* __restrict__ offs,
    u32 const* const* __restrict__ src, u32 const* __restrict__ base, u32* __restrict__ out)
{
  pdl_wait();
  u32 total = offs[nm];
  for (u32 j = blockIdx.x * blockDim.x + threadIdx.x; j < total; j += gridDim.x * blockDim.x) {
    u32 k = find_seg(nm, offs, j);
    u32 const* sk = src[k];
    out[j] = base[k] + (sk ? sk[j - offs[k]] : 0u);
  }
}

// segment of every entity: that of its first vertex
__global__ void k_ent_seg(u32 n, u32 const* __restrict__ voe, u32 vpe,
    u32 const* __restrict__ seg, u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = seg[voe[(size_t)i * vpe]];
}

// per tile of SPLIT_TILE entities (one warp), the count of each segment,
// stored segment-major: hist[seg * ntiles + tile]
__global__ void k_tile_hist(u32 n, u32 const* __restrict__ es, u32 ntiles, u32* __restrict__ hist)
{
  pdl_wait();
  u32 tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (tile >= ntiles) return;
  u32 base = tile * SPLIT_TILE;
  for (u32 c = 0; c < SPLIT_TILE; c += 32) {
    u32 i = base + c + lane;
    bool on = i < n;
    u32 mask = __ballot_sync(FULL_MASK, on);
    if (!mask) break;
    if (on) {
      u32 sg = es[i];
      u32 peers = __match_any_sync(mask, sg);
      if (lane == (u32)(__ffs(peers) - 1)) hist[(size_t)sg * ntiles + tile] += __popc(peers);
    }
    __syncwarp();
  }
}

// stable positions: run[seg * ntiles + tile] starts at the scanned histogram
// and advances as the warp walks its tile in order
__global__ void k_tile_scatter(u32 n, u32 const* __restrict__ es, u32 ntiles, u32* __restrict__ run,
    u32* __restrict__ perm)
{
  pdl_wait();
  u32 tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (tile >= ntiles) return;
  u32 base = tile * SPLIT_TILE;
  u32 lt = (1u << lane) - 1u;
  for (u32 c = 0; c < SPLIT_TILE; c += 32) {
    u32 i = base + c + lane;
    bool on = i < n;
    u32 mask = __ballot_sync(FULL_MASK, on);
    if (!mask) break;
    if (on) {
      u32 sg = es[i];
      u32 peers = __match_any_sync(mask, sg);
      u32 leader = (u32)(__ffs(peers) - 1);
      size_t slot = (size_t)sg * ntiles + tile;
      u32 b = 0;
      if (lane == leader) b = run[slot];
      b = __shfl_sync(peers, b, leader);
      perm[i] = b + __popc(peers & lt);
      if (lane == leader) run[slot] = b + __popc(peers);
    }
    __syncwarp();
  }
}

// first position of every segment (and the total at [nseg])
__global__ void k_seg_bases(u32 nseg, u32 ntiles, u32 const* __restrict__ scan,
    u32* __restrict__ out)
{
  pdl_wait();
  u32 s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s <= nseg) out[s] = scan[(size_t)s * ntiles];
}

__global__ void k_local_ids(u32 n, u32 const* __restrict__ es, u32 const* __restrict__ perm,
    u32 const* __restrict__ bases, u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = perm[i] - bases[es[i]];
}

// dst[seg][local * width + k] = in[i * width + k], vertex ids mapped through
// vloc when given
template <class T>
__global__ void k_scatter_meshes(u32 n, u32 width, T const* __restrict__ in,
    u32 const* __restrict__ es, u32 const* __restrict__ local, u32 const* __restrict__ vloc,
    T* const* __restrict__ dst)
{
  pdl_wait();
  u64 total = (u64)n * width;
  for (u64 j = blockIdx.x * (u64)blockDim.x + threadIdx.x; j < total;
       j += (u64)gridDim.x * blockDim.x) {
    u32 i = (u32)(j / width), k = (u32)(j - (u64)i * width);
    T* d = dst[es[i]];
    if (!d) continue;  // a segment the caller does not want back
    T v = in[j];
    if (vloc) v = (T)vloc[(u32)v];
    d[(u64)local[i] * width + k] = v;
  }
}

// per-segment minimum of element qualities (order-preserving keys)
__global__ void k_seg_min_quality(u32 n, double const* __restrict__ q,
    u32 const* __restrict__ voe, u32 vpe, u32 const* __restrict__ seg,
    unsigned long long* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  bool on = i < n;
  u32 mask = __ballot_sync(FULL_MASK, on);
  if (!on) return;
  u32 sg = seg[voe[(size_t)i * vpe]];
  unsigned long long key = order_key(q[i]);
  u32 peers = __match_any_sync(mask, sg);
  if (peers == FULL_MASK) {
    for (int o = 16; o; o >>= 1) {
      unsigned long long other = __shfl_xor_sync(FULL_MASK, key, o);
      key = other < key ? other : key;
    }
    if ((threadIdx.x & 31) == 0) atomicMin(&out[sg], key);
  } else {
    atomicMin(&out[sg], key);
  }
}

// per-segment count of elements
__global__ void k_seg_count(u32 n, u32 const* __restrict__ voe, u32 vpe,
    u32 const* __restrict__ seg, u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  bool on = i < n;
  u32 mask = __ballot_sync(FULL_MASK, on);
  if (!on) return;
  u32 sg = seg[voe[(size_t)i * vpe]];
  u32 peers = __match_any_sync(mask, sg);
  if ((threadIdx.x & 31) == (u32)(__ffs(peers) - 1)) atomicAdd(&out[sg], (u32)__popc(peers));
}

// small device arrays of pointers / offsets built on the host, uploaded at once
struct Meta {
  std::vector<u64> words;
  size_t add(void const* const* p, u32 n)
  {
    size_t at = words.size();
    for (u32 i = 0; i < n; ++i) words.push_back((u64)(uintptr_t)p[i]);
    return at;
  }
  size_t add_u32(u32 const* p, u32 n)
  {
    size_t at = words.size();
    words.resize(at + (n + 1) / 2, 0);
    std::memcpy(words.data() + at, p, sizeof(u32) * n);
    return at;
  }
  size_t add_u64(u64 const* p, u32 n)
  {
    size_t at = words.size();
    words.insert(words.end(), p, p + n);
    return at;
  }
  u64* dev = nullptr;
  void upload(cudaStream_t s)
  {
    dev = dalloc<u64>(words.size() ? words.size() : 1, s);
    if (!words.empty())
      CK(cudaMemcpyAsync(dev, words.data(), sizeof(u64) * words.size(), cudaMemcpyHostToDevice, s));
  }
  template <class T>
  T* at(size_t w) const
  {
    return reinterpret_cast<T*>(dev + w);
  }
};

template <class T>
void launch_concat(u32 nm, Meta const& meta, size_t src_at, size_t offs_at, u32 width,
    T const* add, u64 total, void* out, cudaStream_t s)
{
  if (!total) return;
  CK(launch_kernel(k_concat<T>, dim3(capped_grid(total)), dim3(BLOCK), 0, s, nm, meta.at<T const* const>(src_at),
      meta.at<u32 const>(offs_at), width, add, static_cast<T*>(out)));
  CK_LAUNCH();
}

template <class T>
void launch_scatter(u32 n, u32 width, void const* in, u32 const* es, u32 const* local,
    u32 const* vloc, Meta const& meta, size_t dst_at, cudaStream_t s)
{
  u64 total = (u64)n * width;
  if (!total) return;
  CK(launch_kernel(k_scatter_meshes<T>, dim3(capped_grid(total)), dim3(BLOCK), 0, s, n, width, static_cast<T const*>(in),
      es, local, vloc, meta.at<T* const>(dst_at)));
  CK_LAUNCH();
}

// Element coordinates are a by-product of collapses (coarsen_transfer adds
// them to the new mesh); every pass recomputes or drops them, so a union
// leaves them out and a mesh leaving it gets them back if its own passes
// would have left them.
bool skipped_tag(Mesh const& m, u32 d, Tag const& t)
{
  return d == m.dim && t.name == "coordinates";
}

// the same tags (names, types, widths) on dimension d, in any order; the
// transfer kind may differ (refinement resets it on vertex fields), each
// mesh's own is restored when it leaves the union
bool same_tags(Mesh& a, Mesh& b, u32 d)
{
  size_t na = 0, nb = 0;
  for (Tag const& x : a.tags[d]) {
    if (skipped_tag(a, d, x)) continue;
    ++na;
    Tag const* y = b.find_tag(d, x.name.c_str());
    if (!y || x.type != y->type || x.ncomps != y->ncomps) return false;
  }
  for (Tag const& y : b.tags[d])
    if (!skipped_tag(b, d, y)) ++nb;
  return na == nb;
}

}  // namespace

Mesh* concat_meshes(std::vector<Mesh*> const& ms)
{
  return concat_meshes(ms, nullptr);
}

void check_batchable(std::vector<Mesh*> const& ms)
{
  if (ms.empty()) throw Failure(E_ARG, "a batch needs at least one mesh");
  Mesh& a = *ms[0];
  u32 dim = a.dim;
  for (Mesh* m : ms) {
    if (m->dim != dim || m->full != a.full || m->parallel != a.parallel)
      throw Failure(E_ARG, "batched meshes differ in dimension, representation or parallelism");
    if (!m->full) throw Failure(E_ARG, "batched meshes need the full representation");
    for (Tag const& t : m->tags[0])
      if (t.type != T_F64 && t.name != "class_dim" && t.name != "class_id")
        throw Failure(E_ARG, "batched meshes may carry only f64 fields and class labels on "
                             "vertices (refinement drops other vertex tags)");
    for (u32 d = 0; d <= dim; ++d) {
      if (m->has_dim(d) != a.has_dim(d) || !same_tags(*m, a, d))
        throw Failure(E_ARG, "batched meshes differ in their entities or tags");
      if (a.parallel && m->has_globals(d) != a.has_globals(d))
        throw Failure(E_ARG, "batched meshes differ in their global numbers");
    }
  }
}

Mesh* concat_meshes(std::vector<Mesh*> const& ms, cudaStream_t stream)
{
  if (ms.empty()) throw Failure(E_ARG, "a batch needs at least one mesh");
  Mesh& a = *ms[0];
  u32 nm = (u32)ms.size(), dim = a.dim;
  // identity numbers in every input stay the identity in the union; other
  // inputs' numbers are written out (on their own streams, before the sync)
  bool iota_glob[4] = {true, true, true, true};
  for (Mesh* m : ms)
    for (u32 d = 0; d < 4; ++d) iota_glob[d] = iota_glob[d] && !m->globals[d];
  for (Mesh* m : ms) {
    if (m->dim != dim || m->full != a.full || m->parallel != a.parallel)
      throw Failure(E_ARG, "batched meshes differ in dimension, representation or parallelism");
    if (!m->full) throw Failure(E_ARG, "batched meshes need the full representation");
    for (Tag const& t : m->tags[0])
      if (t.type != T_F64 && t.name != "class_dim" && t.name != "class_id")
        throw Failure(E_ARG, "batched meshes may carry only f64 fields and class labels on "
                             "vertices (refinement drops other vertex tags)");
    for (u32 d = 0; d <= dim; ++d) {
      if (m->has_dim(d) != a.has_dim(d) || !same_tags(*m, a, d))
        throw Failure(E_ARG, "batched meshes differ in their entities or tags");
      if (a.parallel && m->has_globals(d) != a.has_globals(d))
        throw Failure(E_ARG, "batched meshes differ in their global numbers");
    }
  }
  for (Mesh* m : ms) {
    if (a.parallel)
      for (u32 d = 0; d <= dim; ++d)
        if (!iota_glob[d]) m->ask_globals(d);
    stream_sync(m->s);
  }
  Mesh* u = new Mesh(dim, a.full, a.parallel, stream);
  u->fp32_filter = a.fp32_filter;
  cudaStream_t s = u->s;
  try {
    Meta meta;
    std::vector<u32> offs[4];
    size_t offs_at[4] = {0, 0, 0, 0}, goff_at[4] = {0, 0, 0, 0};
    for (u32 d = 0; d <= dim; ++d) {
      if (!a.has_dim(d)) continue;
      offs[d].assign(nm + 1, 0);
      u64 total = 0;
      for (u32 k = 0; k < nm; ++k) {
        total += ms[k]->counts[d];
        if (total * deg(d, 0) >= (1ull << 32))
          throw Failure(E_ARG, "a union of these meshes exceeds 32-bit entity ids");
        offs[d][k + 1] = (u32)total;
      }
      offs_at[d] = meta.add_u32(offs[d].data(), nm + 1);
      std::vector<u64> g(offs[d].begin(), offs[d].end() - 1);
      goff_at[d] = meta.add_u64(g.data(), nm);
    }
    // source pointers: connectivity, then each tag, then globals
    std::vector<void const*> p(nm);
    size_t conn_at[4] = {0, 0, 0, 0}, glob_at[4] = {0, 0, 0, 0};
    std::vector<size_t> tag_at[4];
    for (u32 d = 0; d <= dim; ++d) {
      if (!a.has_dim(d)) continue;
      if (d) {
        for (u32 k = 0; k < nm; ++k) p[k] = ms[k]->down[d][0];
        conn_at[d] = meta.add(p.data(), nm);
      }
      for (size_t t = 0; t < a.tags[d].size(); ++t) {
        if (skipped_tag(a, d, a.tags[d][t])) {
          tag_at[d].push_back(0);
          continue;
        }
        for (u32 k = 0; k < nm; ++k) p[k] = ms[k]->find_tag(d, a.tags[d][t].name.c_str())->data;
        tag_at[d].push_back(meta.add(p.data(), nm));
      }
      if (a.parallel && a.has_globals(d) && !iota_glob[d]) {
        for (u32 k = 0; k < nm; ++k) p[k] = ms[k]->globals[d];
        glob_at[d] = meta.add(p.data(), nm);
      }
    }
    // segments: one per plain input, all of an input union's
    std::vector<u32> segbase(nm + 1, 0);
    for (u32 k = 0; k < nm; ++k) {
      p[k] = ms[k]->seg;
      segbase[k + 1] = segbase[k] + (ms[k]->seg ? ms[k]->nseg : 1u);
    }
    size_t segsrc_at = meta.add(p.data(), nm);
    size_t segbase_at = meta.add_u32(segbase.data(), nm + 1);
    meta.upload(s);
    for (u32 d = 0; d <= dim; ++d) {
      if (!a.has_dim(d)) continue;
      u32 n = offs[d][nm];
      u32* conn = nullptr;
      if (d) {
        u32 vpe = deg(d, 0);
        conn = dalloc<u32>((size_t)n * vpe, s);
        launch_concat<u32>(nm, meta, conn_at[d], offs_at[d], vpe,
            meta.at<u32 const>(offs_at[0]), (u64)n * vpe, conn, s);
      }
      u->set_ents(d, n, conn);
      for (size_t t = 0; t < a.tags[d].size(); ++t) {
        Tag const& tg = a.tags[d][t];
        if (skipped_tag(a, d, tg)) continue;
        u32 esz = tag_esz(tg.type);
        void* data = dev_alloc((size_t)n * tg.ncomps * esz, s);
        u64 total = (u64)n * tg.ncomps;
        if (esz == 1)
          launch_concat<unsigned char>(nm, meta, tag_at[d][t], offs_at[d], tg.ncomps, nullptr,
              total, data, s);
        else if (esz == 4)
          launch_concat<u32>(nm, meta, tag_at[d][t], offs_at[d], tg.ncomps, nullptr, total,
              data, s);
        else
          launch_concat<u64>(nm, meta, tag_at[d][t], offs_at[d], tg.ncomps, nullptr, total,
              data, s);
        u->add_tag(d, tg.type, tg.name.c_str(), tg.ncomps, tg.transfer, data);
      }
      if (a.parallel && a.has_globals(d) && iota_glob[d]) {
        u->set_iota_globals(d);
      } else if (a.parallel && a.has_globals(d)) {
        u64* g = dalloc<u64>(n, s);
        launch_concat<u64>(nm, meta, glob_at[d], offs_at[d], 1, meta.at<u64 const>(goff_at[d]),
            n, g, s);
        u->set_globals(d, g);
      }
    }
    u->nseg = segbase[nm];
    u32 nv = offs[0][nm];
    u->seg = dalloc<u32>(nv, s);
    if (nv) {
      CK(launch_kernel(k_seg_concat, dim3(capped_grid(nv)), dim3(BLOCK), 0, s, nm, meta.at<u32 const>(offs_at[0]),
          meta.at<u32 const* const>(segsrc_at), meta.at<u32 const>(segbase_at), u->seg));
      CK_LAUNCH();
    }
    dev_free(meta.dev, s);
  } catch (...) {
    delete u;
    throw;
  }
  return u;
}

std::vector<Mesh*> split_union(Mesh& u, cudaStream_t stream)
{
  return split_union(u, stream, nullptr);
}

std::vector<Mesh*> split_union(Mesh& u, cudaStream_t stream, std::vector<char> const* want)
{
  cudaStream_t s = u.s;
  u32 nm = u.nseg, dim = u.dim;
  if (!u.seg) throw Failure(E_ARG, "mesh is not a union of meshes");
  std::vector<Mesh*> out(nm, nullptr);
  u32* es[4] = {};
  u32* local[4] = {};
  std::vector<u32> counts[4];
  try {
    for (u32 k = 0; k < nm; ++k)
      if (!want || (*want)[k]) {
        out[k] = new Mesh(dim, u.full, u.parallel, stream, u.mb);
        out[k]->fp32_filter = u.fp32_filter;
      }
    // stable counting sort of every dimension's entities by segment
    for (u32 d = 0; d <= dim; ++d) {
      if (!u.has_dim(d)) continue;
      u32 n = u.count(d);
      if (d) {
        es[d] = dalloc<u32>(n ? n : 1, s);
        if (n) {
          CK(launch_kernel(k_ent_seg, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, u.ask_down(d, 0), deg(d, 0), u.seg, es[d]));
          CK_LAUNCH();
        }
      } else {
        es[0] = u.seg;
      }
      u32 ntiles = n ? ceil_div(n, SPLIT_TILE) : 1;
      u64 nh = (u64)nm * ntiles;
      if (nh >= (1ull << 32) - 1) throw Failure(E_ARG, "too many meshes in one union to split");
      u32* hist = dalloc<u32>(nh, s);
      CK(cudaMemsetAsync(hist, 0, sizeof(u32) * nh, s));
      u32 warps_per_block = BLOCK / 32;
      if (n) {
        CK(launch_kernel(k_tile_hist, dim3(ceil_div(ntiles, warps_per_block)), dim3(BLOCK), 0, s, n, es[d], ntiles, hist));
        CK_LAUNCH();
      }
      u32* scan = exscan_new(hist, (u32)nh, s);
      dev_free(hist, s);
      u32* bases = dalloc<u32>(nm + 1, s);
      CK(launch_kernel(k_seg_bases, dim3(grid_for(nm + 1)), dim3(BLOCK), 0, s, nm, ntiles, scan, bases));
      CK_LAUNCH();
      u32* perm = dalloc<u32>(n ? n : 1, s);
      if (n) {
        CK(launch_kernel(k_tile_scatter, dim3(ceil_div(ntiles, warps_per_block)), dim3(BLOCK), 0, s, n, es[d], ntiles,
            scan, perm));
        CK_LAUNCH();
      }
      dev_free(scan, s);
      local[d] = dalloc<u32>(n ? n : 1, s);
      if (n) {
        CK(launch_kernel(k_local_ids, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, es[d], perm, bases, local[d]));
        CK_LAUNCH();
      }
      dev_free(perm, s);
      counts[d].resize(nm + 1);
      CK(cudaMemcpyAsync(counts[d].data(), bases, sizeof(u32) * (nm + 1), cudaMemcpyDeviceToHost, s));
      dev_free(bases, s);
    }
    stream_sync(s);
    for (u32 d = 0; d <= dim; ++d) {
      if (!u.has_dim(d)) continue;
      std::vector<u32>& c = counts[d];
      for (u32 k = nm; k > 0; --k) c[k] -= c[k - 1];  // bases -> per-segment counts at [1..nm]
    }
    // allocate every mesh's arrays, then one scatter launch per array
    Meta meta;
    size_t conn_at[4] = {0, 0, 0, 0};
    std::vector<size_t> tag_at[4];
    std::vector<void const*> p(nm);
    for (u32 d = 0; d <= dim; ++d) {
      if (!u.has_dim(d)) continue;
      if (d) {
        u32 vpe = deg(d, 0);
        for (u32 k = 0; k < nm; ++k) {
          p[k] = nullptr;
          if (!out[k]) continue;
          u32 nk = counts[d][k + 1];
          u32* conn = dalloc<u32>((size_t)nk * vpe, s);
          out[k]->set_ents(d, nk, conn);
          p[k] = conn;
        }
        conn_at[d] = meta.add(p.data(), nm);
      } else {
        for (u32 k = 0; k < nm; ++k)
          if (out[k]) out[k]->set_ents(0, counts[0][k + 1], nullptr);
      }
      for (Tag const& t : u.tags[d]) {
        for (u32 k = 0; k < nm; ++k) {
          p[k] = nullptr;
          if (!out[k]) continue;
          u32 nk = counts[d][k + 1];
          void* data = dev_alloc((size_t)nk * t.ncomps * tag_esz(t.type), s);
          out[k]->add_tag(d, t.type, t.name.c_str(), t.ncomps, t.transfer, data);
          p[k] = data;
        }
        tag_at[d].push_back(meta.add(p.data(), nm));
      }
      // each mesh's global numbers restart at 0: its local indices
      if (u.parallel && u.has_globals(d))
        for (u32 k = 0; k < nm; ++k)
          if (out[k]) out[k]->set_iota_globals(d);
    }
    meta.upload(s);
    for (u32 d = 0; d <= dim; ++d) {
      if (!u.has_dim(d)) continue;
      u32 n = u.count(d);
      if (d) launch_scatter<u32>(n, deg(d, 0), u.down[d][0], es[d], local[d], local[0], meta,
          conn_at[d], s);
      for (size_t t = 0; t < u.tags[d].size(); ++t) {
        Tag const& tg = u.tags[d][t];
        u32 esz = tag_esz(tg.type);
        if (esz == 1)
          launch_scatter<unsigned char>(n, tg.ncomps, tg.data, es[d], local[d], nullptr, meta,
              tag_at[d][t], s);
        else if (esz == 4)
          launch_scatter<u32>(n, tg.ncomps, tg.data, es[d], local[d], nullptr, meta,
              tag_at[d][t], s);
        else
          launch_scatter<u64>(n, tg.ncomps, tg.data, es[d], local[d], nullptr, meta,
              tag_at[d][t], s);
      }
    }
    stream_sync(s);
    dev_free(meta.dev, s);
  } catch (...) {
    for (Mesh* m : out) delete m;
    for (u32 d = 1; d < 4; ++d) dev_free(es[d], s);
    for (u32 d = 0; d < 4; ++d) dev_free(local[d], s);
    throw;
  }
  for (u32 d = 1; d < 4; ++d) dev_free(es[d], s);
  for (u32 d = 0; d < 4; ++d) dev_free(local[d], s);
  stream_sync(s);
  return out;
}

// ---------------------------------------------------------------------------
// the per-mesh pass loop over a union

namespace {

__global__ void k_seg_min_quality(u32 n, double const* __restrict__ q,
    u32 const* __restrict__ voe, u32 vpe, u32 const* __restrict__ seg,
    unsigned long long* __restrict__ out);
__global__ void k_seg_count(u32 n, u32 const* __restrict__ voe, u32 vpe,
    u32 const* __restrict__ seg, u32* __restrict__ out);

}  // namespace

UnionCtl::UnionCtl(Mesh& m) : u(m), nm(m.nseg)
{
  cudaStream_t s = u.s;
  active = dalloc<u32>(nm, s);
  floor = dalloc<double>(nm, s);
  selected = dalloc<u32>(nm, s);
  elems = dalloc<u32>(nm, s);
  minkey = dalloc<unsigned long long>(nm, s);
  CK(cudaMallocHost(&h_u32, sizeof(u32) * 2 * nm));
  CK(cudaMallocHost(&h_key, sizeof(unsigned long long) * nm));
}

UnionCtl::~UnionCtl()
{
  cudaStream_t s = u.s;
  u.ctl = nullptr;
  cudaStreamSynchronize(s);
  dev_free(active, s);
  dev_free(floor, s);
  dev_free(selected, s);
  dev_free(elems, s);
  dev_free(minkey, s);
  cudaFreeHost(h_u32);
  cudaFreeHost(h_key);
}

std::vector<double> UnionCtl::min_quality()
{
  cudaStream_t s = u.s;
  u32 ne = u.count(u.dim);
  double const* q = u.qualities();
  CK(cudaMemsetAsync(minkey, 0xff, sizeof(unsigned long long) * nm, s));
  if (ne) {
    CK(launch_kernel(k_seg_min_quality, dim3(grid_for(ne)), dim3(BLOCK), 0, s, ne, q, u.ask_down(u.dim, 0),
        deg(u.dim, 0), u.seg, minkey));
    CK_LAUNCH();
  }
  CK(cudaMemcpyAsync(h_key, minkey, sizeof(unsigned long long) * nm, cudaMemcpyDeviceToHost, s));
  stream_sync(s);
  std::vector<double> r(nm);
  for (u32 k = 0; k < nm; ++k) r[k] = h_key[k] == ~0ull ? DBL_MAX : from_order_key(h_key[k]);
  return r;
}

void UnionCtl::run(u32 op, std::vector<u32> const& group, std::vector<double> const& floors,
    double size_floor, double good_qual, u32 nlayers)
{
  cudaStream_t s = u.s;
  std::vector<u32> act(nm, 0);
  for (u32 k : group) act[k] = 1;
  CK(cudaMemcpyAsync(active, act.data(), sizeof(u32) * nm, cudaMemcpyHostToDevice, s));
  bool with_floor = op == OP_REFINE || op == OP_COARSEN;
  if (with_floor)
    CK(cudaMemcpyAsync(floor, floors.data(), sizeof(double) * nm, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(selected, 0, sizeof(u32) * nm, s));
  CK(cudaMemsetAsync(elems, 0, sizeof(u32) * nm, s));
  u32 ne = u.count(u.dim);
  if (ne) {
    CK(launch_kernel(k_seg_count, dim3(grid_for(ne)), dim3(BLOCK), 0, s, ne, u.ask_down(u.dim, 0), deg(u.dim, 0), u.seg,
        elems));
    CK_LAUNCH();
  }
  ctl.active = active;
  ctl.floor = with_floor ? floor : nullptr;
  ctl.selected = selected;
  u.ctl = &ctl;
  try {
    switch (op) {
      case OP_REFINE: refine_by_size(u, 0.0); break;
      case OP_COARSEN: coarsen_by_size(u, 0.0, size_floor); break;
      case OP_SWAP: swap_slivers(u, good_qual, nlayers); break;
      default: coarsen_slivers(u, good_qual, nlayers); break;
    }
  } catch (...) {
    u.ctl = nullptr;
    throw;
  }
  u.ctl = nullptr;
  CK(cudaMemcpyAsync(h_u32, selected, sizeof(u32) * nm, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(h_u32 + nm, elems, sizeof(u32) * nm, cudaMemcpyDeviceToHost, s));
  stream_sync(s);
  last_batch_stats().union_passes += 1;
}

namespace {

double wall_s()
{
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// consecutive runs of `idx` whose current elements sum to at most `max`
// (0 = no limit); each run holds at least one mesh
std::vector<std::vector<u32>> chunks_of(std::vector<Mesh*>& ms, std::vector<u32> const& idx,
    unsigned long long max)
{
  std::vector<std::vector<u32>> out;
  std::vector<u32> cur;
  unsigned long long sum = 0;
  for (u32 k : idx) {
    unsigned long long ne = ms[k]->count(ms[k]->dim);
    if (!cur.empty() && max && sum + ne > max) {
      out.push_back(cur);
      cur.clear();
      sum = 0;
    }
    cur.push_back(k);
    sum += ne;
  }
  if (!cur.empty()) out.push_back(cur);
  return out;
}

}  // namespace

bool GroupRunner::step(std::vector<Mesh*>& ms, std::vector<SegState>& st,
    std::vector<char>& owned)
{
  BatchStats& bs = last_batch_stats();
  u32 n = (u32)ms.size();
  bool live = false;
  for (u32 k = 0; k < n; ++k) live = live || st[k].state < ST_DONE;
  if (!live) return false;
  bs.steps += 1;
  auto group = [&](u32 state) {
    std::vector<u32> g;
    for (u32 k = 0; k < n; ++k)
      if (st[k].state == state) g.push_back(k);
    return g;
  };
  // incr_op_count (adapt.cpp:36-45) for mesh k after a pass that changed it
  auto counted = [&](u32 k, u32 op, u32 elems) {
    BatchMeshResult& r = st[k].res;
    r.ops.push_back(op);
    r.passes += 1;
    r.changed = 1;
    r.elems_in += elems;
    bs.mesh_passes += 1;
    bs.elems_in += elems;
    if (st[k].ops > ap.max_ops) {
      r.status = E_MAXOPS;
      st[k].state = ST_FAILED;
      return;
    }
    ++st[k].ops;
  };
  auto replace = [&](u32 k, Mesh* m) {
    if (owned[k]) delete ms[k];
    ms[k] = m;
    owned[k] = 1;
  };
  // a union of the meshes c; a lone mesh is its own union of one segment,
  // changed in place by the pass with nothing to copy in or out
  auto gather = [&](std::vector<u32> const& c) {
    if (c.size() == 1) {
      Mesh* m = ms[c[0]];
      if (!m->seg) {
        u32 nv = m->count(0);
        m->seg = dalloc<u32>(nv ? nv : 1, m->s);
        CK(cudaMemsetAsync(m->seg, 0, sizeof(u32) * (nv ? nv : 1), m->s));
        m->nseg = 1;
      }
      return m;
    }
    std::vector<Mesh*> parts;
    for (u32 k : c) parts.push_back(ms[k]);
    bs.unions += 1;
    double t = wall_s();
    Mesh* u = concat_meshes(parts, s);
    stream_sync(s);
    bs.secs_concat += wall_s() - t;
    return u;
  };
  auto release = [&](Mesh* u, std::vector<u32> const& c) {
    if (c.size() != 1) delete u;
  };
  auto split = [&](Mesh& u, std::vector<char> const& want) {
    double t = wall_s();
    std::vector<Mesh*> o = split_union(u, s, &want);
    bs.secs_split += wall_s() - t;
    return o;
  };
  // satisfy_size's floor (adapt.cpp:47-52), once per mesh
  for (auto const& c : chunks_of(ms, group(ST_INIT), max_union_elems)) {
    Mesh* u = gather(c);
    std::vector<double> mq;
    try {
      UnionCtl ctl(*u);
      mq = ctl.min_quality();
    } catch (...) {
      release(u, c);
      throw;
    }
    release(u, c);
    for (u32 j = 0; j < c.size(); ++j) {
      SegState& x = st[c[j]];
      x.qf = mq[j];
      if (ap.good_qual < x.qf) x.qf = ap.good_qual;
      x.state = ST_REFINE;
    }
  }
  // satisfy_size: refine while it changes a mesh, then coarsen
  for (u32 op : {OP_REFINE, OP_COARSEN}) {
    u32 here = op == OP_REFINE ? ST_REFINE : ST_COARSEN;
    u32 next = op == OP_REFINE ? ST_COARSEN : ST_SHAPE;
    for (auto const& c : chunks_of(ms, group(here), max_union_elems)) {
      Mesh* u = gather(c);
      u32 m = (u32)c.size();
      std::vector<u32> sel(m), elems(m), all(m);
      std::vector<double> qf(m);
      for (u32 j = 0; j < m; ++j) {
        all[j] = j;
        qf[j] = st[c[j]].qf;
      }
      std::vector<Mesh*> outs;
      try {
        {
          double t = wall_s();
          UnionCtl ctl(*u);
          ctl.run(op, all, qf, ap.size_floor, ap.good_qual, ap.nlayers);
          bs.secs_passes += wall_s() - t;
          for (u32 j = 0; j < m; ++j) {
            sel[j] = ctl.h_u32[j];
            elems[j] = ctl.h_u32[m + j];
          }
        }
        if (m > 1) {
          std::vector<char> want(m);
          for (u32 j = 0; j < m; ++j) want[j] = sel[j] ? 1 : 0;
          outs = split(*u, want);
        }
      } catch (...) {
        release(u, c);
        throw;
      }
      release(u, c);
      for (u32 j = 0; j < m; ++j) {
        u32 k = c[j];
        if (sel[j]) {
          counted(k, op, elems[j]);
          if (m > 1) replace(k, outs[j]);
        } else {
          st[k].state = next;
        }
      }
    }
  }
  // satisfy_shape (adapt.cpp:58-80): swap, else collapse slivers
  for (auto const& c : chunks_of(ms, group(ST_SHAPE), max_union_elems)) {
    Mesh* u = gather(c);
    u32 m = (u32)c.size();
    std::vector<char> changed(m, 0);
    std::vector<Mesh*> outs;
    try {
      double t = wall_s();
      UnionCtl ctl(*u);
      std::vector<double> mq = ctl.min_quality(), qf(m, 0.0);
      std::vector<u32> g2, g3;
      for (u32 j = 0; j < m; ++j)
        if (mq[j] >= ap.good_qual)
          st[c[j]].state = ST_DONE;
        else
          g2.push_back(j);
      if (u->dim == 3 && !g2.empty()) {
        ctl.run(OP_SWAP, g2, qf, ap.size_floor, ap.good_qual, ap.nlayers);
        for (u32 j : g2)
          if (ctl.h_u32[j]) {
            counted(c[j], OP_SWAP, ctl.h_u32[m + j]);
            changed[j] = 1;
          } else {
            g3.push_back(j);
          }
      } else {
        g3 = g2;
      }
      if (!g3.empty()) {
        ctl.run(OP_CSLIVERS, g3, qf, ap.size_floor, ap.good_qual, ap.nlayers);
        for (u32 j : g3)
          if (ctl.h_u32[j]) {
            counted(c[j], OP_CSLIVERS, ctl.h_u32[m + j]);
            changed[j] = 1;
          } else {
            st[c[j]].state = ST_DONE;  // shape quality could not be satisfied
          }
      }
      bs.secs_passes += wall_s() - t;
    } catch (...) {
      release(u, c);
      throw;
    }
    bool any = false;
    for (char x : changed) any = any || x;
    if (any && m > 1) {
      try {
        outs = split(*u, changed);
      } catch (...) {
        release(u, c);
        throw;
      }
      for (u32 j = 0; j < m; ++j)
        if (changed[j]) replace(c[j], outs[j]);
    }
    release(u, c);
  }
  live = false;
  for (u32 k = 0; k < n; ++k) live = live || st[k].state < ST_DONE;
  return live;
}

// ---------------------------------------------------------------------------
// content digest: an order-sensitive 64-bit hash of every array of a mesh

namespace {

__device__ inline u64 mix64(u64 z)
{
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// sum over words of mix(word, position, salt); wraps modulo 2^64
__global__ void k_digest(u64 nwords, u32 const* __restrict__ w, u64 salt, u64* out)
{
  pdl_wait();
  u64 acc = 0;
  for (u64 j = blockIdx.x * (u64)blockDim.x + threadIdx.x; j < nwords;
       j += (u64)gridDim.x * blockDim.x)
    acc += mix64(((u64)w[j] << 32) ^ mix64(j + salt));
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(FULL_MASK, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd((unsigned long long*)out, (unsigned long long)acc);
}

u64 host_mix(u64 z)
{
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

u64 str_hash(std::string const& x)
{
  u64 h = 1469598103934665603ull;
  for (unsigned char c : x) h = (h ^ c) * 1099511628211ull;
  return h;
}

}  // namespace

u64 mesh_digest(Mesh& m)
{
  cudaStream_t s = m.s;
  u64* acc = dalloc<u64>(1, s);
  CK(cudaMemsetAsync(acc, 0, sizeof(u64), s));
  u64 h = host_mix(m.dim);
  u64 salt = 0;
  auto add = [&](void const* p, u64 bytes) {
    salt = host_mix(salt + 1);
    u64 nw = bytes / 4;
    if (nw) {
      CK(launch_kernel(k_digest, dim3(capped_grid(nw)), dim3(BLOCK), 0, s, nw, static_cast<u32 const*>(p), salt, acc));
      CK_LAUNCH();
    }
    // a trailing partial word (u8 tags) enters through the host
    if (bytes % 4) {
      unsigned char tail[4] = {0, 0, 0, 0};
      CK(cudaMemcpyAsync(tail, static_cast<unsigned char const*>(p) + nw * 4, bytes % 4,
          cudaMemcpyDeviceToHost, s));
      stream_sync(s);
      u32 t;
      std::memcpy(&t, tail, 4);
      h = host_mix(h ^ t ^ salt);
    }
  };
  for (u32 d = 0; d <= m.dim; ++d) {
    if (!m.has_dim(d)) continue;
    u32 n = m.count(d);
    h = host_mix(h ^ (((u64)d << 32) | n));
    if (d) add(m.ask_down(d, 0), (u64)n * deg(d, 0) * 4);
    for (Tag const& t : m.tags[d]) {
      h = host_mix(h ^ str_hash(t.name) ^ ((u64)t.type << 40) ^ ((u64)t.ncomps << 20) ^ t.transfer);
      add(t.data, (u64)n * t.ncomps * tag_esz(t.type));
    }
    if (m.has_globals(d)) add(m.ask_globals(d), (u64)n * 8);
  }
  u64 dev = 0;
  CK(cudaMemcpyAsync(&dev, acc, sizeof(u64), cudaMemcpyDeviceToHost, s));
  stream_sync(s);
  dev_free(acc, s);
  return host_mix(h ^ dev);
}

// ---------------------------------------------------------------------------
// tag lists: which tags a pass leaves on each dimension, and in what order.
// A union's tag list follows the passes the union ran; each mesh's must
// follow the passes that changed it, so the split replays those.

namespace {

Tag const* find_in(std::vector<Tag> const& v, char const* name)
{
  for (Tag const& t : v)
    if (t.name == name) return &t;
  return nullptr;
}

}  // namespace

Layout layout_of(Mesh& m)
{
  Layout l;
  for (u32 d = 0; d <= m.dim; ++d)
    for (Tag const& t : m.tags[d]) {
      Tag x = t;
      x.data = nullptr;
      l.tags[d].push_back(x);
    }
  return l;
}

// the tag lists refine_build, coarsen_build and swap_build produce
Layout layout_after(u32 op, Layout const& in, u32 dim)
{
  Layout out;
  std::vector<Tag> cls;
  if (find_in(in.tags[0], "class_dim")) {
    for (char const* nm : {"class_dim", "class_id"})
      for (u32 d = 0; d <= dim; ++d)
        if (Tag const* t = find_in(in.tags[d], nm)) {
          if (d == 0) {
            Tag x = *t;
            cls.push_back(x);
          }
        }
  }
  auto class_of = [&](u32 d) {
    std::vector<Tag> v;
    for (Tag const& c : cls)
      if (Tag const* t = find_in(in.tags[d], c.name.c_str())) v.push_back(*t);
    return v;
  };
  // vertices: refinement keeps the f64 fields, then the class labels;
  // collapses and swaps keep every vertex tag in place
  if (op == OP_REFINE) {
    for (Tag const& t : in.tags[0])
      if (t.type == T_F64) {
        Tag x = t;
        x.transfer = X_NOT;  // refine_build re-adds vertex fields untransferred
        out.tags[0].push_back(x);
      }
    for (Tag const& t : class_of(0)) out.tags[0].push_back(t);
  } else {
    out.tags[0] = in.tags[0];
  }
  for (u32 d = 1; d <= dim; ++d) {
    out.tags[d] = class_of(d);
    if (d != dim) continue;
    for (Tag const& t : in.tags[d])
      if (t.type == T_F64 && t.transfer == X_CONSERVE) out.tags[d].push_back(t);
    bool any_fit = false;
    for (Tag const& t : in.tags[d])
      if (t.type == T_F64 && t.transfer == X_POINTWISE) any_fit = true;
    if (any_fit && (op == OP_COARSEN || op == OP_CSLIVERS)) {
      Tag x;
      x.name = "coordinates";
      x.type = T_F64;
      x.ncomps = 3;
      x.transfer = X_NOT;
      out.tags[d].push_back(x);
    }
    for (Tag const& t : in.tags[d])
      if (t.type == T_F64 && t.transfer == X_POINTWISE) out.tags[d].push_back(t);
  }
  return out;
}

// give mesh m exactly the tags of `want`, in its order: element coordinates
// (which a collapse leaves behind) are recomputed when wanted, dropped when not
void apply_layout(Mesh& m, Layout const& want)
{
  u32 dim = m.dim;
  if (m.find_tag(dim, "coordinates")) m.remove_tag(dim, "coordinates");
  if (find_in(want.tags[dim], "coordinates")) interp_coords_to_elems(m);
  for (u32 d = 0; d <= dim; ++d) {
    std::vector<Tag> next;
    for (Tag const& w : want.tags[d]) {
      Tag* t = m.find_tag(d, w.name.c_str());
      if (!t) throw Failure(E_ARG, "batched mesh lost tag " + w.name);
      next.push_back(*t);
      next.back().transfer = w.transfer;
      t->data = nullptr;
    }
    for (Tag& t : m.tags[d]) dev_free(t.data, m.s);
    m.tags[d].swap(next);
  }
}

void drop_segments(Mesh& m)
{
  dev_free(m.seg, m.s);
  m.seg = nullptr;
  m.nseg = 0;
}

void adapt_batch(std::vector<Mesh*> const& ms, double size_floor, double good_qual,
    u32 nlayers, u32 max_ops, unsigned long long max_union_elems,
    std::vector<BatchMeshResult>& res)
{
  last_batch_stats() = BatchStats();
  u32 n = (u32)ms.size();
  res.assign(n, BatchMeshResult());
  if (!n) return;
  check_batchable(ms);
  for (Mesh* m : ms) stream_sync(m->s);
  GroupRunner run;
  run.ap = AdaptParams{size_floor, good_qual, nlayers, max_ops};
  run.max_union_elems = max_union_elems;
  CK(cudaStreamCreateWithFlags(&run.s, cudaStreamNonBlocking));
  std::vector<Mesh*> cur(ms.begin(), ms.end());
  std::vector<char> owned(n, 0);
  std::vector<SegState> st(n);
  std::vector<Layout> start(n);
  for (u32 k = 0; k < n; ++k) start[k] = layout_of(*ms[k]);
  auto cleanup = [&]() {
    for (u32 k = 0; k < n; ++k)
      if (owned[k]) delete cur[k];
    release_stream_scratch(run.s);
    cudaStreamSynchronize(run.s);
    cudaStreamDestroy(run.s);
  };
  try {
    while (run.step(cur, st, owned)) {
    }
    stream_sync(run.s);
    for (u32 k = 0; k < n; ++k) {
      res[k] = st[k].res;
      drop_segments(*cur[k]);
      if (!st[k].res.passes) continue;  // no pass changed this mesh
      Layout want = start[k];
      for (u32 op : st[k].res.ops) want = layout_after(op, want, ms[k]->dim);
      apply_layout(*cur[k], want);
      if (!owned[k]) continue;  // changed in place
      stream_sync(cur[k]->s);
      ms[k]->overwrite(cur[k]);
      owned[k] = 0;
    }
  } catch (...) {
    cleanup();
    throw;
  }
  cleanup();
}

}  // namespace osh
