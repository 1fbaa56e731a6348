// Mesh store, lazy adjacency derivation and per-element geometry on sm_100a.
//
// Adjacency kernels (all one pass over their inputs, no host round trips
// except where an output size must be known to allocate):
//   up_from_down   counting by atomics, one scan, atomic fill, then a
//                  warp-per-row rank sort that restores the deterministic
//                  row order of the reference's CPU invert_map
//                  (invert_map.cpp:92-136) and splits use -> (high, dir)
//   reflect_down   one thread per (high entity, local low slot); searches the
//                  first vertex's upward list (reflect_down.cpp:13-38,
//                  find_by_verts.hpp:14-55)
//   dual / stars   star.cpp, dual.cpp, bridge_graph.cpp, derive_sides.cpp
#include <cfloat>
#include <cmath>
#include <cstring>

#include "mesh.hpp"

namespace osh {

// ---------------------------------------------------------------------------
// Mesh lifetime and tags

static void release_mailbox(Mailbox* m)
{
  m->release();
  delete m;
}

Mesh::Mesh(u32 d, bool f, bool p, cudaStream_t stream,
    std::shared_ptr<Mailbox> mailbox, bool exact_stream)
    : dim(d), full(f), parallel(p), s(stream), mb(mailbox)
{
  if (!s && !exact_stream) {
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    own_stream = true;
  }
  if (!mb) {
    mb = std::shared_ptr<Mailbox>(new Mailbox(), release_mailbox);
    mb->init(s);
  }
}

Mesh::~Mesh()
{
  try {
    clear_contents();
  } catch (...) {
  }
  if (own_stream) {
    mb.reset();
    release_stream_scratch(s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
}

Mesh* Mesh::spawn() const
{
  // the same stream as this mesh, the legacy default stream included
  Mesh* m = new Mesh(dim, full, parallel, s, mb, true);
  m->nseg = nseg;
  m->ctl = ctl;
  m->fp32_filter = fp32_filter;
  return m;
}

Mesh* Mesh::clone()
{
  Mesh* c = new Mesh(dim, full, parallel, nullptr);
  stream_sync(s);
  try {
    for (u32 d = 0; d <= dim; ++d) {
      if (!has_dim(d)) continue;
      u32 n = counts[d];
      u32* v = nullptr;
      if (d) {
        size_t bytes = sizeof(u32) * (size_t)n * deg(d, 0);
        v = static_cast<u32*>(dev_alloc(bytes, c->s));
        CK(cudaMemcpyAsync(v, down[d][0], bytes, cudaMemcpyDeviceToDevice, c->s));
      }
      c->set_ents(d, n, v);
      for (auto const& t : tags[d]) {
        size_t bytes = (size_t)n * t.ncomps * tag_esz(t.type);
        void* p = dev_alloc(bytes, c->s);
        CK(cudaMemcpyAsync(p, t.data, bytes, cudaMemcpyDeviceToDevice, c->s));
        c->add_tag(d, t.type, t.name.c_str(), t.ncomps, t.transfer, p);
      }
      if (globals[d]) {
        u64* g = dalloc<u64>(n, c->s);
        CK(cudaMemcpyAsync(g, globals[d], sizeof(u64) * n, cudaMemcpyDeviceToDevice, c->s));
        c->globals[d] = g;
      }
      c->globals_iota[d] = globals_iota[d];
      c->ranks_zero[d] = ranks_zero[d];
      c->ids_iota[d] = ids_iota[d];
      u32* const* own[2] = {&own_ranks[d], &own_ids[d]};
      u32** cown[2] = {&c->own_ranks[d], &c->own_ids[d]};
      for (u32 k = 0; k < 2; ++k)
        if (*own[k]) {
          *cown[k] = dalloc<u32>(n ? n : 1, c->s);
          CK(cudaMemcpyAsync(*cown[k], *own[k], sizeof(u32) * n, cudaMemcpyDeviceToDevice,
              c->s));
        }
    }
    c->ghost_layers = ghost_layers;
    c->fp32_filter = fp32_filter;
    if (seg) {
      c->nseg = nseg;
      c->seg = dalloc<u32>(counts[0], c->s);
      CK(cudaMemcpyAsync(c->seg, seg, sizeof(u32) * counts[0], cudaMemcpyDeviceToDevice,
          c->s));
    }
    stream_sync(c->s);
  } catch (...) {
    delete c;
    throw;
  }
  return c;
}

void Mesh::own_new_stream()
{
  stream_sync(s);
  if (own_stream) return;
  CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  own_stream = true;
  mb = std::shared_ptr<Mailbox>(new Mailbox(), release_mailbox);
  mb->init(s);
}

void Mesh::use_stream(cudaStream_t stream)
{
  stream_sync(s);
  if (own_stream) {
    release_stream_scratch(s);
    CK(cudaStreamDestroy(s));
  }
  own_stream = false;
  s = stream;
}

void Mesh::clear_contents()
{
  for (u32 h = 0; h < 4; ++h)
    for (u32 l = 0; l < 4; ++l) {
      dev_free(down[h][l], s);
      down[h][l] = nullptr;
      if (have_up[l][h]) {
        dev_free(up[l][h].offs, s);
        dev_free(up[l][h].adj, s);
        dev_free(up[l][h].dirs, s);
        dev_free(up[l][h].pre, s);
        up[l][h] = UpAdj();
        have_up[l][h] = false;
        up_sorted[l][h] = false;
      }
      if (have_star[l][h]) {
        dev_free(star[l][h].offs, s);
        dev_free(star[l][h].adj, s);
        star[l][h] = Graph();
        have_star[l][h] = false;
      }
    }
  dev_free(dual, s);
  dual = nullptr;
  for (u32 d = 0; d < 3; ++d) {
    dev_free(low_row_offs[d], s);
    dev_free(low_rows[d], s);
    low_row_offs[d] = nullptr;
    low_rows[d] = nullptr;
  }
  search_marks = nullptr;  // the stream's, not the mesh's
  for (u32 d = 0; d < 4; ++d) {
    for (auto& t : tags[d]) dev_free(t.data, s);
    tags[d].clear();
    dev_free(globals[d], s);
    globals[d] = nullptr;
    dev_free(own_ranks[d], s);
    own_ranks[d] = nullptr;
    dev_free(own_ids[d], s);
    own_ids[d] = nullptr;
    globals_iota[d] = ranks_zero[d] = ids_iota[d] = false;
    counts[d] = 0;
  }
  dev_free(qual_cache, s);
  qual_cache = nullptr;
  dev_free(seg, s);
  seg = nullptr;
}

void Mesh::overwrite(Mesh* with)
{
  clear_contents();
  dim = with->dim;
  full = with->full;
  parallel = with->parallel;
  for (u32 h = 0; h < 4; ++h)
    for (u32 l = 0; l < 4; ++l) {
      down[h][l] = with->down[h][l];
      up[h][l] = with->up[h][l];
      have_up[h][l] = with->have_up[h][l];
      up_sorted[h][l] = with->up_sorted[h][l];
      star[h][l] = with->star[h][l];
      have_star[h][l] = with->have_star[h][l];
      with->down[h][l] = nullptr;
      with->have_up[h][l] = false;
      with->have_star[h][l] = false;
    }
  dual = with->dual;
  with->dual = nullptr;
  for (u32 d = 0; d < 3; ++d) {
    low_row_offs[d] = with->low_row_offs[d];
    low_rows[d] = with->low_rows[d];
    with->low_row_offs[d] = nullptr;
    with->low_rows[d] = nullptr;
  }
  search_marks = with->search_marks;
  search_gen = with->search_gen;
  with->search_marks = nullptr;
  for (u32 d = 0; d < 4; ++d) {
    counts[d] = with->counts[d];
    tags[d].swap(with->tags[d]);
    globals[d] = with->globals[d];
    with->globals[d] = nullptr;
    own_ranks[d] = with->own_ranks[d];
    with->own_ranks[d] = nullptr;
    own_ids[d] = with->own_ids[d];
    with->own_ids[d] = nullptr;
    globals_iota[d] = with->globals_iota[d];
    ranks_zero[d] = with->ranks_zero[d];
    ids_iota[d] = with->ids_iota[d];
  }
  ghost_layers = with->ghost_layers;
  qual_cache = with->qual_cache;
  with->qual_cache = nullptr;
  nseg = with->nseg;
  seg = with->seg;
  with->seg = nullptr;
  delete with;
}

void Mesh::set_ents(u32 d, u32 n, u32* verts)
{
  counts[d] = n;
  down[d][0] = verts;
}

u32 Mesh::count(u32 d)
{
  if (d > dim) return 0;
  if (d) ask_down(d, 0);
  return counts[d];
}

Tag* Mesh::find_tag(u32 d, char const* name)
{
  for (auto& t : tags[d])
    if (t.name == name) return &t;
  return nullptr;
}

Tag& Mesh::add_tag(u32 d, u32 type, char const* name, u32 ncomps, u32 transfer,
    void* data)
{
  if (find_tag(d, name)) throw Failure(E_ARG, std::string("duplicate tag ") + name);
  Tag t;
  t.name = name;
  t.type = type;
  t.ncomps = ncomps;
  t.transfer = transfer;
  t.data = data;
  tags[d].push_back(t);
  return tags[d].back();
}

void Mesh::remove_tag(u32 d, char const* name)
{
  for (size_t i = 0; i < tags[d].size(); ++i)
    if (tags[d][i].name == name) {
      dev_free(tags[d][i].data, s);
      tags[d].erase(tags[d].begin() + i);
      return;
    }
  throw Failure(E_ARG, std::string("no tag ") + name);
}

double const* Mesh::coords()
{
  Tag* t = find_tag(0, "coordinates");
  if (!t) throw Failure(E_ARG, "mesh has no coordinates");
  return static_cast<double const*>(t->data);
}

void Mesh::set_globals(u32 d, u64* g)
{
  dev_free(globals[d], s);
  globals[d] = g;
  globals_iota[d] = false;
  dev_free(own_ranks[d], s);
  own_ranks[d] = nullptr;
  ranks_zero[d] = false;
  dev_free(own_ids[d], s);
  own_ids[d] = nullptr;
  ids_iota[d] = false;
}

void Mesh::set_iota_globals(u32 d)
{
  set_globals(d, nullptr);
  globals_iota[d] = true;
}

u64 const* Mesh::ask_globals(u32 d)
{
  if (!globals[d] && globals_iota[d]) {
    u32 n = count(d);
    globals[d] = dalloc<u64>(n ? n : 1, s);
    iota_u64(globals[d], n, s);
  }
  return globals[d];
}

u32 const* Mesh::ask_own_ranks(u32 d)
{
  if (!own_ranks[d] && ranks_zero[d]) {
    u32 n = count(d);
    own_ranks[d] = dalloc<u32>(n ? n : 1, s);
    fill_u32(own_ranks[d], n, 0, s);
  }
  return own_ranks[d];
}

u32 const* Mesh::ask_own_ids(u32 d)
{
  if (!own_ids[d] && ids_iota[d]) {
    u32 n = count(d);
    own_ids[d] = dalloc<u32>(n ? n : 1, s);
    iota_u32(own_ids[d], n, 1, s);
  }
  return own_ids[d];
}

void Mesh::ensure_ghosting(u32 nlayers)
{
  if (!parallel || seg || nlayers == ghost_layers) return;
  // unghost_mesh / ghost_mesh rebuild the mesh: owners are forgotten, and
  // ghosting tags the owner ranks of every dimension it holds
  for (u32 d = 0; d < 4; ++d) {
    dev_free(own_ranks[d], s);
    own_ranks[d] = nullptr;
    dev_free(own_ids[d], s);
    own_ids[d] = nullptr;
    ids_iota[d] = false;
    ranks_zero[d] = nlayers && d <= dim && has_dim(d);
  }
  ghost_layers = nlayers;
}

void Mesh::note_exchange(u32 d)
{
  if (!parallel || seg || d > dim) return;
  if (!own_ranks[d]) ranks_zero[d] = true;
  if (!own_ids[d]) ids_iota[d] = true;
}

void Mesh::make_parallel()
{
  parallel = true;
  for (u32 d = 0; d <= dim; ++d)
    if (has_dim(d)) set_iota_globals(d);
}

// ---------------------------------------------------------------------------
// upward adjacency (up_from_down.cpp:24-47, invert_map.cpp:70-136)

__global__ void k_count_lows(u32 const* __restrict__ loh, u32 nuses, u32* cnt)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nuses) atomicAdd(&cnt[loh[i]], 1u);
}

// cnt holds each row's count: a row's uses take its slots from the end down
// (their order is arbitrary either way; the rows are ranked or marked
// unsorted afterwards), so no cursor array is zeroed for the fill
__global__ void k_fill_uses(u32 const* __restrict__ loh, u32 nuses,
    u32 const* __restrict__ offs, u32* cnt, u32* __restrict__ tmp)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nuses) return;
  u32 l = loh[i];
  u32 slot = atomicSub(&cnt[l], 1u) - 1u;
  tmp[offs[l] + slot] = i;
}

// One warp per row: every lane ranks its element against the whole row and
// writes it to its sorted position (rows hold distinct use indices).
__global__ void k_rank_rows(u32 const* __restrict__ offs, u32 const* __restrict__ tmp,
    u32 nrows, u32 lph, u32* __restrict__ adj, u32* __restrict__ dirs)
{
  pdl_wait();
  u32 row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  u32 lane = threadIdx.x & 31;
  if (row >= nrows) return;
  u32 f = offs[row], len = offs[row + 1] - f;
  for (u32 base = 0; base < len; base += 32) {
    u32 idx = base + lane;
    u32 my = idx < len ? tmp[f + idx] : INV;
    u32 rank = 0;
    for (u32 cb = 0; cb < len; cb += 32) {
      u32 other = (cb + lane < len) ? tmp[f + cb + lane] : INV;
      u32 lim = len - cb < 32 ? len - cb : 32;
      for (u32 j = 0; j < lim; ++j) {
        u32 v = __shfl_sync(0xffffffffu, other, j);
        rank += (v < my) ? 1u : 0u;
      }
    }
    if (idx < len) {
      adj[f + rank] = my / lph;
      dirs[f + rank] = my % lph;
    }
  }
}

// Each row (the uses of one low entity, filled in arbitrary order) is
// sorted by a group of G lanes holding K elements each: a bitonic network
// over N = G*K slots in registers, partners across lanes exchanged by
// shuffles, the missing slots padded with the largest key. Rows longer than
// N (rare: N is at least 2.5x the mean degree) are ranked by the group from
// global memory after the network, outside any shuffle.
template <int G, int K>
__global__ void __launch_bounds__(256)
k_sort_rows(u32 const* __restrict__ offs, u32 const* __restrict__ pre,
    u32 const* __restrict__ tmp, u32 nrows, u32 lph, u32* __restrict__ adj,
    u32* __restrict__ dirs)
{
  pdl_wait();
  constexpr int N = G * K;
  u32 row = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  u32 l = threadIdx.x % G;
  u32 f = 0, len = 0;
  if (row < nrows) {
    f = offs[row] + (pre ? pre[row] : 0u);
    len = offs[row + 1] - f;
  }
  u32 v[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    u32 idx = k * G + l;
    v[k] = (idx < len && len <= (u32)N) ? tmp[f + idx] : 0xffffffffu;
  }
#pragma unroll
  for (int size = 2; size <= N; size <<= 1) {
#pragma unroll
    for (int j = size >> 1; j > 0; j >>= 1) {
      u32 nv[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        u32 i = k * G + l;
        u32 other = (j < G) ? __shfl_xor_sync(0xffffffffu, v[k], j) : v[k ^ (j / G)];
        bool up = (i & size) == 0;
        bool lower = (i & j) == 0;
        u32 mn = v[k] < other ? v[k] : other;
        u32 mx = v[k] < other ? other : v[k];
        nv[k] = (lower == up) ? mn : mx;
      }
#pragma unroll
      for (int k = 0; k < K; ++k) v[k] = nv[k];
    }
  }
  if (len <= (u32)N) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      u32 idx = k * G + l;
      if (idx < len) {
        adj[f + idx] = v[k] / lph;
        dirs[f + idx] = v[k] % lph;
      }
    }
  } else {
    for (u32 a = l; a < len; a += G) {
      u32 x = tmp[f + a], rank = 0;
      for (u32 b = 0; b < len; ++b) rank += (tmp[f + b] < x) ? 1u : 0u;
      adj[f + rank] = x / lph;
      dirs[f + rank] = x % lph;
    }
  }
}

template <int G, int K>
static void launch_sort_rows(u32 const* offs, u32 const* pre, u32 const* tmp, u32 nrows,
    u32 lph, u32* adj, u32* dirs, cudaStream_t s)
{
  u64 threads = (u64)nrows * G;
  CK(launch_kernel(k_sort_rows<G, K>, dim3(grid_for(threads)), dim3(256), 0, s, offs, pre, tmp, nrows, lph, adj, dirs));
  CK_LAUNCH();
}

// sort every row (or, given pre, every row's part after its first pre[l]
// uses); nsort = the uses to be sorted in all
static void rank_rows(u32 const* offs, u32 const* pre, u32 const* tmp, u32 nrows, u32 nsort,
    u32 lph, u32* adj, u32* dirs, cudaStream_t s)
{
  double avg = nrows ? (double)nsort / nrows : 1.0;
  double want = 2.5 * avg;
  if (want <= 2) launch_sort_rows<2, 1>(offs, pre, tmp, nrows, lph, adj, dirs, s);
  else if (want <= 4) launch_sort_rows<4, 1>(offs, pre, tmp, nrows, lph, adj, dirs, s);
  else if (want <= 8) launch_sort_rows<8, 1>(offs, pre, tmp, nrows, lph, adj, dirs, s);
  else if (want <= 16) launch_sort_rows<16, 1>(offs, pre, tmp, nrows, lph, adj, dirs, s);
  else if (want <= 32) launch_sort_rows<32, 1>(offs, pre, tmp, nrows, lph, adj, dirs, s);
  else if (want <= 64) launch_sort_rows<32, 2>(offs, pre, tmp, nrows, lph, adj, dirs, s);
  else launch_sort_rows<32, 4>(offs, pre, tmp, nrows, lph, adj, dirs, s);
}

// as k_fill_uses, the row's slots taken from its end down
__global__ void k_fill_uses_split(u32 const* __restrict__ loh, u32 nuses, u32 lph,
    u32 const* __restrict__ offs, u32* cnt, u32* __restrict__ adj, u32* __restrict__ dirs)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nuses) return;
  u32 l = loh[i];
  u32 slot = offs[l] + atomicSub(&cnt[l], 1u) - 1u;
  adj[slot] = i / lph;
  dirs[slot] = i % lph;
}

__global__ void k_join_uses(u32 n, u32 lph, u32 const* __restrict__ adj,
    u32 const* __restrict__ dirs, u32* __restrict__ uses)
{
  pdl_wait();
  u32 j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) uses[j] = adj[j] * lph + dirs[j];
}

void up_from_down_unsorted(u32 high, u32 low, u32 nhighs, u32 nlows, u32 const* loh,
    UpAdj& out, cudaStream_t s)
{
  u32 lph = deg(high, low);
  u32 nuses = nhighs * lph;
  u32* cnt = dalloc<u32>((size_t)nlows + 1, s);
  CK(cudaMemsetAsync(cnt, 0, sizeof(u32) * ((size_t)nlows + 1), s));
  if (nuses) {
    PROBE(P_UP_COUNT, s, 4.0 * nuses + 4.0 * nlows);
    CK(launch_kernel(k_count_lows, dim3(grid_for(nuses)), dim3(BLOCK), 0, s, loh, nuses, cnt));
    CK_LAUNCH();
  }
  out.offs = exscan_new(cnt, nlows, s);
  out.adj = dalloc<u32>(nuses, s);
  out.dirs = dalloc<u32>(nuses, s);
  if (nuses) {
    PROBE(P_UP_FILL, s, 4.0 * nuses + 4.0 * (nlows + 1.0) + 4.0 * nlows + 8.0 * nuses);
    CK(launch_kernel(k_fill_uses_split, dim3(grid_for(nuses)), dim3(BLOCK), 0, s, loh, nuses, lph, out.offs, cnt,
        out.adj, out.dirs));
    CK_LAUNCH();
  }
  dev_free(cnt, s);
}

// the packed uses of each row's part after its first pre[l] (the part the
// sort reorders), a thread per row: a carried row's tail holds only the
// uses of the entities the pass made, so most rows have none
__global__ void k_join_tails(u32 nlows, u32 lph, u32 const* __restrict__ offs,
    u32 const* __restrict__ pre, u32 const* __restrict__ adj, u32 const* __restrict__ dirs,
    u32* __restrict__ uses)
{
  pdl_wait();
  for (u32 l = blockIdx.x * blockDim.x + threadIdx.x; l < nlows; l += gridDim.x * blockDim.x)
    for (u32 p = offs[l] + pre[l], e = offs[l + 1]; p < e; ++p) uses[p] = adj[p] * lph + dirs[p];
}

void sort_up_rows(u32 high, u32 low, u32 nhighs, u32 nlows, UpAdj const& u,
    cudaStream_t s)
{
  u32 lph = deg(high, low);
  u32 nuses = nhighs * lph;
  if (!nuses || !nlows) return;
  u32* uses = dalloc<u32>(nuses, s);
  if (u.pre) {
    CK(launch_kernel(k_join_tails, dim3(std::min<u32>(grid_for(nlows), 148u * 8u)),
        dim3(BLOCK), 0, s, nlows, lph, u.offs, u.pre, u.adj, u.dirs, uses));
  } else {
    CK(launch_kernel(k_join_uses, dim3(grid_for(nuses)), dim3(BLOCK), 0, s, nuses, lph, u.adj,
        u.dirs, uses));
  }
  CK_LAUNCH();
  {
    u32 nsort = u.pre ? nuses - u.npre : nuses;
    PROBE(P_UP_RANK, s, 12.0 * nsort + 4.0 * (nlows + 1.0));
    rank_rows(u.offs, u.pre, uses, nlows, nsort, lph, u.adj, u.dirs, s);
  }
  dev_free(uses, s);
}

void up_from_down(u32 high, u32 low, u32 nhighs, u32 nlows, u32 const* loh,
    UpAdj& out, cudaStream_t s)
{
  u32 lph = deg(high, low);
  u32 nuses = nhighs * lph;
  u32* cnt = dalloc<u32>((size_t)nlows + 1, s);
  CK(cudaMemsetAsync(cnt, 0, sizeof(u32) * ((size_t)nlows + 1), s));
  if (nuses) {
    PROBE(P_UP_COUNT, s, 4.0 * nuses + 4.0 * nlows);
    CK(launch_kernel(k_count_lows, dim3(grid_for(nuses)), dim3(BLOCK), 0, s, loh, nuses, cnt));
    CK_LAUNCH();
  }
  out.offs = exscan_new(cnt, nlows, s);
  u32* tmp = dalloc<u32>(nuses, s);
  out.adj = dalloc<u32>(nuses, s);
  out.dirs = dalloc<u32>(nuses, s);
  if (nuses) {
    {
      PROBE(P_UP_FILL, s, 8.0 * nuses + 4.0 * (nlows + 1.0) + 4.0 * nlows);
      CK(launch_kernel(k_fill_uses, dim3(grid_for(nuses)), dim3(BLOCK), 0, s, loh, nuses, out.offs, cnt, tmp));
      CK_LAUNCH();
    }
    if (nlows) {
      PROBE(P_UP_RANK, s, 12.0 * nuses + 4.0 * (nlows + 1.0));
      rank_rows(out.offs, nullptr, tmp, nlows, nuses, lph, out.adj, out.dirs, s);
    }
  }
  dev_free(tmp, s);
  dev_free(cnt, s);
}

// ---------------------------------------------------------------------------
// downward adjacency by search (reflect_down.cpp:13-81)

// reflect_down_entity / find_by_verts (reflect_down.cpp:13-38,
// find_by_verts.hpp:14-76): the low entity with the wanted vertices is
// unique, so it is found among the entities that share its smallest vertex,
// where every low entity is listed once with its other vertices. Each
// vertex's entities are split over SUB sub-rows by a hash of their other
// vertices (4 for edges, 8 for triangles), so a search reads about 1/SUB of
// the vertex's row: the vertices a refinement left with the lowest ids are
// the smallest vertex of most entities around them, and a single
// tet-to-triangle search of a refined 2M-tet mesh took 254 us scanning their
// whole rows. Consecutive entities mostly share their smallest vertex, so
// the fill's writes stay close together (a hash of the whole tuple over all
// buckets scattered them and made the fill slower than the search it
// saved). A row's order does not matter: a search reads a whole sub-row and
// the key is unique.

__device__ inline void sort_small(u32* w, u32 n)
{
  for (u32 i = 1; i < n; ++i)
    for (u32 j = i; j > 0 && w[j - 1] > w[j]; --j) {
      u32 t = w[j];
      w[j] = w[j - 1];
      w[j - 1] = t;
    }
}

template <u32 VPL>
struct KeyRows {
  static constexpr u32 SUB = VPL == 2 ? 4 : 8;
};

// sub-row of a sorted tuple: its smallest vertex's SUB sub-rows, picked by
// murmur3's 32-bit finaliser over the other vertices
template <u32 VPL>
__device__ inline u32 key_row(u32 const* w)
{
  u32 h = w[1] * 0x9e3779b1u + (VPL == 3 ? w[2] * 0x85ebca77u : 0u);
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return w[0] * KeyRows<VPL>::SUB + (h & (KeyRows<VPL>::SUB - 1));
}

template <u32 VPL>
__device__ inline void low_key(u32 const* __restrict__ vol, u32 i, u32* w)
{
#pragma unroll
  for (u32 k = 0; k < VPL; ++k) w[k] = vol[(size_t)i * VPL + k];
  sort_small(w, VPL);
}

// The rows of the edges (low 1) and the triangles (low 2) are built in the
// same launches when both are needed (blockIdx.y: the job). marks
// (optional): only entities whose smallest vertex is marked are listed.
struct KeyJob {
  u32 low, nl;
  u32 const* vol;
  u32* cnt;
  u32 const* offs;
  u32* rows;
};
struct KeyJobs {
  KeyJob j[2];
};

template <u32 VPL>
__device__ inline void count_key_row(KeyJob const jb, u32 i, u32 const* __restrict__ marks,
    u32 gen)
{
  u32 w[VPL];
  low_key<VPL>(jb.vol, i, w);
  if (marks && marks[w[0]] != gen) return;
  atomicAdd(&jb.cnt[key_row<VPL>(w)], 1u);
}

// (grid-stride: with marks most threads read a vertex tuple and leave)
__global__ void k_count_key_rows(const __grid_constant__ KeyJobs jobs,
    u32 const* __restrict__ marks, u32 gen)
{
  pdl_wait();
  KeyJob const jb = jobs.j[blockIdx.y];
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < jb.nl; i += gridDim.x * blockDim.x) {
    if (jb.low == 1)
      count_key_row<2>(jb, i, marks, gen);
    else
      count_key_row<3>(jb, i, marks, gen);
  }
}

// cnt holds each sub-row's count; a row's records take its slots from the
// end down: uint2 {v1, id} for edges, uint4 {v1, v2, id, 0} for triangles
template <u32 VPL>
__device__ inline void fill_key_row(KeyJob const jb, u32 i, u32 const* __restrict__ marks,
    u32 gen)
{
  u32 w[VPL];
  low_key<VPL>(jb.vol, i, w);
  if (marks && marks[w[0]] != gen) return;
  u32 b = key_row<VPL>(w);
  u32 slot = jb.offs[b] + atomicSub(&jb.cnt[b], 1u) - 1u;
  if (VPL == 2)
    reinterpret_cast<uint2*>(jb.rows)[slot] = make_uint2(w[1], i);
  else
    reinterpret_cast<uint4*>(jb.rows)[slot] = make_uint4(w[1], w[VPL - 1], i, 0u);
}

__global__ void k_fill_key_rows(const __grid_constant__ KeyJobs jobs,
    u32 const* __restrict__ marks, u32 gen)
{
  pdl_wait();
  KeyJob const jb = jobs.j[blockIdx.y];
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < jb.nl; i += gridDim.x * blockDim.x) {
    if (jb.low == 1)
      fill_key_row<2>(jb, i, marks, gen);
    else
      fill_key_row<3>(jb, i, marks, gen);
  }
}

// One thread per high entity: every wanted low's sub-row bounds are loaded
// together, then each sub-row is read four records at a time. The
// searches of a pass's pairs share a launch (blockIdx.y: the pair).
struct ReflectJob {
  u32 high, low, first, nh;
  u32 const* voh;
  u32 const* offs;
  u32 const* rows;
  u32* out;
};
struct ReflectJobs {
  ReflectJob j[3];
};

template <u32 HIGH, u32 LOW>
__device__ inline void reflect_keyed(ReflectJob const jb, u32 i)
{
  constexpr u32 LPH = HIGH == 3 ? (LOW == 1 ? 6 : 4) : 3;
  constexpr u32 VPH = HIGH + 1, VPL = LOW + 1;
  u32 const* __restrict__ voh = jb.voh;
  u32 const* __restrict__ offs = jb.offs;
  u32 const* __restrict__ rows = jb.rows;
  u32 v[VPH];
#pragma unroll
  for (u32 k = 0; k < VPH; ++k) v[k] = voh[(size_t)i * VPH + k];
  u32 t[LPH][VPL], f[LPH], e[LPH];
#pragma unroll
  for (u32 j = 0; j < LPH; ++j) {
#pragma unroll
    for (u32 k = 0; k < VPL; ++k) t[j][k] = v[canon(HIGH, LOW, 0, j, k)];
    sort_small(t[j], VPL);
  }
#pragma unroll
  for (u32 j = 0; j < LPH; ++j) {
    u32 b = key_row<VPL>(t[j]);
    f[j] = offs[b];
    e[j] = offs[b + 1];
  }
#pragma unroll
  for (u32 j = 0; j < LPH; ++j) {
    u32 found = INV;
    for (u32 k = f[j]; k < e[j] && found == INV; k += 4) {
      if (LOW == 1) {
        uint2 x[4];
        uint2 const* r = reinterpret_cast<uint2 const*>(rows);
#pragma unroll
        for (u32 q = 0; q < 4; ++q) x[q] = k + q < e[j] ? __ldg(r + k + q) : make_uint2(INV, INV);
#pragma unroll
        for (u32 q = 0; q < 4; ++q)
          if (x[q].x == t[j][1]) found = x[q].y;
      } else {
        uint4 x[4];
        uint4 const* r = reinterpret_cast<uint4 const*>(rows);
#pragma unroll
        for (u32 q = 0; q < 4; ++q)
          x[q] = k + q < e[j] ? __ldg(r + k + q) : make_uint4(INV, INV, INV, INV);
#pragma unroll
        for (u32 q = 0; q < 4; ++q)
          if (x[q].x == t[j][1] && x[q].y == t[j][VPL - 1]) found = x[q].z;
      }
    }
    jb.out[(size_t)i * LPH + j] = found;
  }
}

__global__ void k_reflect_keyed(const __grid_constant__ ReflectJobs jobs)
{
  pdl_wait();
  ReflectJob const jb = jobs.j[blockIdx.y];
  u32 i = jb.first + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= jb.nh) return;
  if (jb.high == 2)
    reflect_keyed<2, 1>(jb, i);
  else if (jb.low == 1)
    reflect_keyed<3, 1>(jb, i);
  else
    reflect_keyed<3, 2>(jb, i);
}

// ---------------------------------------------------------------------------
// star graphs (star.cpp)

__global__ void k_vertex_edge_star(u32 nadj, u32 const* __restrict__ adj,
    u32 const* __restrict__ dirs, u32 const* __restrict__ voe, u32* __restrict__ star)
{
  pdl_wait();
  u32 j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nadj) star[j] = voe[adj[j] * 2 + (1 - dirs[j])];
}

__global__ void k_scale_offsets(u32 const* __restrict__ in, u32 n1, u32 k,
    u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n1) out[i] = in[i] * k;
}

__global__ void k_edge_tri_star(u32 nadj, u32 const* __restrict__ adj,
    u32 const* __restrict__ dirs, u32 const* __restrict__ eot, u32* __restrict__ star)
{
  pdl_wait();
  u32 j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nadj) return;
  u32 t = adj[j], d = dirs[j];
  star[j * 2 + 0] = eot[t * 3 + (d + 1) % 3];
  star[j * 2 + 1] = eot[t * 3 + (d + 2) % 3];
}

__global__ void k_sum_degrees(u32 n, u32 const* __restrict__ a, u32 const* __restrict__ b,
    u32* __restrict__ deg_out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) deg_out[i] = (a[i + 1] - a[i]) + (b[i + 1] - b[i]);
}

__global__ void k_edge_tet_star(u32 n, u32 const* __restrict__ so,
    u32 const* __restrict__ ts_offs, u32 const* __restrict__ ts,
    u32 const* __restrict__ roe_offs, u32 const* __restrict__ roe,
    u32 const* __restrict__ roe_dirs, u32 const* __restrict__ eor, u32* __restrict__ star)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 o = so[i];
  for (u32 j = ts_offs[i]; j < ts_offs[i + 1]; ++j) star[o++] = ts[j];
  for (u32 j = roe_offs[i]; j < roe_offs[i + 1]; ++j)
    star[o++] = eor[roe[j] * 6 + tet_opp_edge(roe_dirs[j])];
}

constexpr u32 STAR_BUF = 256;

// get_ent_star_general (star.cpp:14-34); pass 0 counts, pass 1 fills
__global__ void k_star_general(u32 n, u32 const* __restrict__ hl_offs,
    u32 const* __restrict__ hl, u32 const* __restrict__ loh, u32 lph,
    u32 const* __restrict__ star_offs, u32* __restrict__ deg_out,
    u32* __restrict__ star, u32* err)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 buf[STAR_BUF];
  u32 size = 0;
  for (u32 j = hl_offs[i]; j < hl_offs[i + 1]; ++j) {
    u32 h = hl[j];
    for (u32 k = 0; k < lph; ++k) {
      u32 sl = loh[h * lph + k];
      if (sl == i) continue;
      bool have = false;
      for (u32 a = 0; a < size; ++a)
        if (buf[a] == sl) {
          have = true;
          break;
        }
      if (have) continue;
      if (size == STAR_BUF) {
        atomicOr(err, 1u);
        continue;
      }
      buf[size++] = sl;
    }
  }
  if (star)
    for (u32 a = 0; a < size; ++a) star[star_offs[i] + a] = buf[a];
  else
    deg_out[i] = size;
}

// ---------------------------------------------------------------------------
// element dual (dual.cpp)

__global__ void k_dual_from_sides(u32 ne, u32 spe, u32 const* __restrict__ soe,
    u32 const* __restrict__ es_offs, u32 const* __restrict__ es, u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  for (u32 j = 0; j < spe; ++j) {
    u32 s = soe[i * spe + j];
    u32 o = INV;
    for (u32 k = es_offs[s]; k < es_offs[s + 1]; ++k)
      if (es[k] != i) {
        o = es[k];
        break;
      }
    out[i * spe + j] = o;
  }
}

__global__ void k_dual_from_verts(u32 dim, u32 ne, u32 const* __restrict__ voe,
    u32 const* __restrict__ ev_offs, u32 const* __restrict__ ev,
    u32* __restrict__ out, u32* err)
{
  pdl_wait();
  u32 spe = deg(dim, dim - 1), vpe = deg(dim, 0), vps = deg(dim - 1, 0);
  u32 idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ne * spe) return;
  u32 i = idx / spe, j = idx % spe;
  u32 buf[STAR_BUF];
  u32 n = 0;
  for (u32 k = 0; k < vps; ++k) {
    u32 v = voe[(size_t)i * vpe + canon(dim, dim - 1, 0, j, k)];
    u32 f = ev_offs[v], e = ev_offs[v + 1];
    if (k) {
      u32 nn = 0;
      for (u32 a = 0; a < n; ++a) {
        bool has = false;
        for (u32 b = f; b < e; ++b)
          if (ev[b] == buf[a]) {
            has = true;
            break;
          }
        if (has) buf[nn++] = buf[a];
      }
      n = nn;
    } else {
      for (u32 a = f; a < e; ++a)
        if (ev[a] != i) {
          if (n == STAR_BUF) {
            atomicOr(err, 1u);
            break;
          }
          buf[n++] = ev[a];
        }
    }
  }
  out[idx] = n ? buf[0] : INV;
}

// bridge graphs (bridge_graph.cpp): degree then fill
__global__ void k_bridge_degree(u32 n, u32 const* __restrict__ offs, u32 stride,
    u32 const* __restrict__ adj, u32* __restrict__ degree)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 f = offs ? offs[i] : i * stride, e = offs ? offs[i + 1] : (i + 1) * stride;
  u32 d = 0;
  for (u32 j = f; j < e; ++j)
    if (i < adj[j]) ++d;
  degree[i] = d;
}

__global__ void k_bridge_edges(u32 n, u32 const* __restrict__ offs,
    u32 const* __restrict__ adj, u32 const* __restrict__ bo, u32* __restrict__ voe)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 e = bo[i];
  for (u32 j = offs[i]; j < offs[i + 1]; ++j)
    if (i < adj[j]) {
      voe[e * 2 + 0] = i;
      voe[e * 2 + 1] = adj[j];
      ++e;
    }
}

// bridge_dual_graph + derive_side: sides in (element, local side) order
__global__ void k_derive_sides(u32 dim, u32 ne, u32 const* __restrict__ dual,
    u32 const* __restrict__ bo, u32 const* __restrict__ voe, u32* __restrict__ vos)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  u32 spe = deg(dim, dim - 1), vpe = deg(dim, 0), vps = deg(dim - 1, 0);
  u32 s = bo[i];
  for (u32 j = 0; j < spe; ++j)
    if (i < dual[i * spe + j]) {
      for (u32 k = 0; k < vps; ++k)
        vos[(size_t)s * vps + k] = voe[(size_t)i * vpe + canon(dim, dim - 1, 0, j, k)];
      ++s;
    }
}

// ---------------------------------------------------------------------------
// Mesh::ask_* (mesh.cpp:136-261)

// the vertices of high entities first..nh-1 of up to two dimensions
// (blockIdx.y picks one)
struct MarkRange {
  u32 first, nh, vph;
  u32 const* voh;
};
struct MarkRanges {
  MarkRange r[2];
};

__global__ void k_mark_verts(const __grid_constant__ MarkRanges rs, u32* __restrict__ marks,
    u32 gen)
{
  pdl_wait();
  MarkRange const r = rs.r[blockIdx.y];
  u32 i = r.first + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.nh) return;
  for (u32 k = 0; k < r.vph; ++k) marks[r.voh[(size_t)i * r.vph + k]] = gen;
}

// Search rows limited to what a pass's products need: the vertices of the
// high entities from first[h] on (h = 2, 3) are marked, and the rows list
// only the low entities whose smallest vertex is marked (a product's lows
// all have one of its vertices as their smallest). They serve those
// searches only, so drop_search_rows discards them afterwards.
void Mesh::mark_search_verts(u32 const* first)
{
  // the stream's marks, stamped with a generation of their own (nothing to
  // zero between uses)
  u32 nv = counts[0];
  search_marks = stream_marks(KEPT_MARKS, nv ? nv : 1, s, &search_gen);
  MarkRanges rs;
  u32 nr = 0, most = 0;
  for (u32 h = 2; h <= dim; ++h) {
    u32 nh = count(h);
    if (first[h] >= nh) continue;
    rs.r[nr++] = MarkRange{first[h], nh, deg(h, 0), ask_down(h, 0)};
    most = std::max(most, nh - first[h]);
  }
  if (nr) {
    CK(launch_kernel(k_mark_verts, dim3(grid_for(most), nr), dim3(BLOCK), 0, s, rs,
        search_marks, search_gen));
    CK_LAUNCH();
  }
}

void Mesh::drop_search_rows()
{
  if (!search_marks) return;
  for (u32 d = 1; d < 3; ++d) {
    dev_free(low_row_offs[d], s);
    dev_free(low_rows[d], s);
    low_row_offs[d] = nullptr;
    low_rows[d] = nullptr;
  }
  search_marks = nullptr;  // the stream's marks stay for its next use
}

// the search rows of the listed lows (1: edges, 2: triangles) that are
// not built yet, the two built in the same launches
void Mesh::build_low_rows(u32 const* lows, u32 nlows)
{
  KeyJobs jobs;
  u32 nj = 0, most = 0;
  ScanJob sj[2];
  for (u32 q = 0; q < nlows; ++q) {
    u32 low = lows[q];
    if (low_rows[low]) continue;
    u32 const* vol = ask_down(low, 0);
    u32 nl = counts[low];
    size_t nb = (size_t)counts[0] * (low == 1 ? KeyRows<2>::SUB : KeyRows<3>::SUB);
    if (nb >= 0xffffffffull) throw Failure(E_ARG, "reflect_down: too many vertices");
    // counts in the stream's kept scratch, zero on entry: the fill takes
    // every count back down to zero
    u32* cnt = stream_zero_scratch(nj == 0 ? KEPT_ROWS0 : KEPT_ROWS1, nb + 1, s);
    low_row_offs[low] = dalloc<u32>(nb + 1, s);
    low_rows[low] = dalloc<u32>((size_t)nl * (low == 1 ? 2 : 4), s);
    jobs.j[nj] = KeyJob{low, nl, vol, cnt, low_row_offs[low], low_rows[low]};
    sj[nj] = ScanJob{cnt, low_row_offs[low], nullptr, nullptr, (u32)nb, 0};
    most = std::max(most, nl);
    ++nj;
  }
  if (!nj) return;
  if (most) {
    CK(launch_kernel(k_count_key_rows, dim3(std::min<u32>(grid_for(most), 148u * 8u), nj),
        dim3(BLOCK), 0, s, jobs, search_marks, search_gen));
    CK_LAUNCH();
  }
  exscan_jobs(sj, nj, s);
  if (most) {
    CK(launch_kernel(k_fill_key_rows, dim3(std::min<u32>(grid_for(most), 148u * 8u), nj),
        dim3(BLOCK), 0, s, jobs, search_marks, search_gen));
    CK_LAUNCH();
  }
}

// down(high, low) of the high entities first..count(high)-1 of each listed
// pair into outs[q] (the survivors' part is the caller's), one launch
void Mesh::reflect_many(u32 const* highs, u32 const* lows, u32 const* firsts, u32* const* outs,
    u32 npairs)
{
  u32 need[2], nneed = 0;
  for (u32 q = 0; q < npairs; ++q) {
    if (firsts[q] >= count(highs[q])) continue;
    bool have = false;
    for (u32 k = 0; k < nneed; ++k) have = have || need[k] == lows[q];
    if (!have) need[nneed++] = lows[q];
  }
  if (!nneed) return;
  build_low_rows(need, nneed);
  ReflectJobs jobs;
  u32 nj = 0, most = 0;
  double bytes = 0;
  for (u32 q = 0; q < npairs; ++q) {
    u32 high = highs[q], low = lows[q], first = firsts[q], nh = count(high);
    if (first >= nh) continue;
    jobs.j[nj++] = ReflectJob{high, low, first, nh, ask_down(high, 0), low_row_offs[low],
        low_rows[low], outs[q]};
    most = std::max(most, nh - first);
    // voh once, each wanted low's sub-row bounds and its records (a few of
    // 8 / 16 bytes) once, out once
    double n = (double)(nh - first) * deg(high, low), rec = low == 1 ? 8.0 : 16.0;
    bytes += 4.0 * deg(high, 0) * (nh - first) + (8.0 + 4.0 * rec) * n + 4.0 * n;
  }
  PROBE(P_REFLECT_DOWN, s, bytes);
  u32 const gb = tuned(TK_GATHER_BLOCK);
  CK(launch_kernel(k_reflect_keyed, dim3(grid_for(most, gb), nj), dim3(gb), 0, s, jobs));
  CK_LAUNCH();
}

void Mesh::reflect_range(u32 high, u32 low, u32 first, u32* out)
{
  reflect_many(&high, &low, &first, &out, 1);
}

// new ids of a surviving high entity's lows: its old lows through the lows'
// survivor offsets (a surviving entity's lows all survive). A thread takes
// CARRY_UNROLL entries a block apart (reads and writes stay coalesced) and
// issues all their loads before it uses any: the gather through same_l is
// the one random access, and a single entry per thread left the kernel
// waiting on two dependent loads per entry.
constexpr u32 CARRY_UNROLL = 4;

// the carries of a pass's pairs share a launch (blockIdx.y: the pair)
struct DownJob {
  u32 n, lph;
  u32 const* same_h;
  u32 const* same_l;
  u32 const* old_down;
  u32* out;
};
struct DownJobs {
  DownJob j[3];
};

template <u32 LPH>
__device__ inline void carry_down_rows(DownJob const jb)
{
  u32 const* __restrict__ same_h = jb.same_h;
  u32 const* __restrict__ same_l = jb.same_l;
  u32 const* __restrict__ old_down = jb.old_down;
  u32* __restrict__ out = jb.out;
  u32 const n = jb.n, bs = blockDim.x;
  u32 base = blockIdx.x * (bs * CARRY_UNROLL) + threadIdx.x;
  u32 od[CARRY_UNROLL], ni[CARRY_UNROLL], nn[CARRY_UNROLL];
#pragma unroll
  for (u32 k = 0; k < CARRY_UNROLL; ++k) {
    u32 t = base + k * bs;
    od[k] = 0;
    ni[k] = nn[k] = 0;
    if (t < n) {
      u32 i = t / LPH;
      ni[k] = same_h[i];
      nn[k] = same_h[i + 1];
      od[k] = old_down[t];
    }
  }
#pragma unroll
  for (u32 k = 0; k < CARRY_UNROLL; ++k) {
    u32 t = base + k * bs;
    if (t < n && nn[k] != ni[k]) out[(size_t)ni[k] * LPH + t % LPH] = same_l[od[k]];
  }
}

__global__ void __launch_bounds__(512) k_carry_down(const __grid_constant__ DownJobs jobs)
{
  pdl_wait();
  // (the job by value: a reference into the parameters would put the whole
  // job array in local memory)
  DownJob const jb = jobs.j[blockIdx.y];
  if (jb.lph == 3)
    carry_down_rows<3>(jb);
  else if (jb.lph == 4)
    carry_down_rows<4>(jb);
  else
    carry_down_rows<6>(jb);
}

void carry_down_all(Mesh& m, Mesh& out, u32* const* same_of, u32 const* nsame_of)
{
  u32 const dim = m.dim;
  cudaStream_t s = out.s;
  // the pairs carried: the survivors' part in one launch, then the
  // products' part searched in one launch
  u32 hs[3], ls[3], firsts[3];
  u32* dns[3];
  u32 np = 0;
  DownJobs jobs;
  u32 nj = 0;
  u64 most = 0;
  double bytes = 0;
  u64 nprod = 0;
  u32 first[4] = {0, 0, 0, 0};
  for (u32 h = 2; h <= dim; ++h) {
    first[h] = out.has_dim(h) ? out.count(h) : 0;
    for (u32 l = 1; l < h; ++l) {
      if (!same_of[h] || !same_of[l]) continue;
      if (!m.down[h][l] || out.down[h][l] || !out.has_dim(h) || !out.has_dim(l)) continue;
      u32 nh_old = m.counts[h], nh = out.count(h), lph = deg(h, l);
      out.count(l);
      u32* dn = dalloc<u32>((size_t)nh * lph, s);
      if (nh_old) {
        u32 n = nh_old * lph;
        jobs.j[nj++] = DownJob{n, lph, same_of[h], same_of[l], m.down[h][l], dn};
        most = std::max<u64>(most, n);
        bytes += 4.0 * (nh_old + 1) + 12.0 * n;
      }
      hs[np] = h;
      ls[np] = l;
      firsts[np] = nsame_of[h];
      dns[np] = dn;
      ++np;
      first[h] = nsame_of[h];
    }
    nprod += out.has_dim(h) ? out.count(h) - first[h] : 0;
  }
  if (nj) {
    PROBE(P_CARRY, s, bytes);
    u32 const gb = tuned(TK_GATHER_BLOCK);
    u32 g = (u32)ceil_div(most, (u64)gb * CARRY_UNROLL);
    CK(launch_kernel(k_carry_down, dim3(g, nj), dim3(gb), 0, s, jobs));
    CK_LAUNCH();
  }
  // rows limited to the products' vertices when the products touch few
  // enough of them (a quarter of the vertices at most, four per product)
  bool const marked = np && !out.low_rows[1] && !out.low_rows[2] && !out.search_marks &&
      16 * nprod < out.count(0);
  if (marked) out.mark_search_verts(first);
  out.reflect_many(hs, ls, firsts, dns, np);
  if (marked) out.drop_search_rows();
  for (u32 q = 0; q < np; ++q) out.down[hs[q]][ls[q]] = dns[q];
}

// up(low, high) carried through a pass. A surviving low keeps the uses of
// its old row whose high entity survived, in the old order, mapped to new
// ids, followed by the uses of the entities the pass made; a low the pass
// made has only such uses (a surviving high entity's lows all survive).
// On short rows (edges, faces) one thread walks one old row, eight uses at
// a time with their loads issued together; long rows (vertices) take a lane
// group each (the _grouped kernels below). newid_h holds each old high
// entity's new id or INV, one gather per use. The kernel is bound by how
// many rows are in flight, not by the gather. (Measured alternatives: a
// lane group for every row left too few short rows in flight and ran at
// half the speed; a warp per 32 rows reading their uses coalesced ran at
// the same speed as a thread per row; for passes that removed few
// entities, new ids from a shared-memory table of id buckets, on a grid
// capped to the blocks that fit with the table, ran 25% slower; reading a
// row as the 16-byte words that hold it, three per array instead of eight
// loads, took 48 registers and ran 15% slower with fewer blocks resident.)
__global__ void k_new_ids(u32 n, u32 const* __restrict__ same, u32* __restrict__ newid)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 a = same[i];
  newid[i] = same[i + 1] != a ? a : INV;
}

// The uses of the entities the pass made (generated uses first..nuses-1 of
// the new down(high, low), lph per high entity): cnt holds each row's kept +
// generated uses, and the generated ones take the slots after the kept
// ones, from the row's end down (their order within a row is arbitrary
// either way: the rows are marked unsorted). The fill kernels below run
// these on their threads past the old rows, so the two parts of a row's
// fill, which write disjoint slots, share one launch.
struct UpGen {
  u32 first, nuses, lph;
  u32 const* loh;
  u32* cnt;
};

__device__ inline void up_gen_fill(UpGen const& g, u32 k, u32 const* __restrict__ offs,
    u32* __restrict__ adj, u32* __restrict__ dirs)
{
  u32 const u = g.first + k;
  if (u >= g.nuses) return;
  u32 l = g.loh[u];
  u32 slot = offs[l] + atomicSub(&g.cnt[l], 1u) - 1u;
  adj[slot] = u / g.lph;
  dirs[slot] = u % g.lph;
}

constexpr u32 FILL_BATCH = 8;

__global__ void k_up_surv_fill(u32 nl_old, u32 const* __restrict__ same_l,
    u32 const* __restrict__ newid_h, u32 const* __restrict__ offs_old,
    u32 const* __restrict__ adj_old, u32 const* __restrict__ dirs_old,
    u32 const* __restrict__ offs, u32* __restrict__ adj, u32* __restrict__ dirs, UpGen gen)
{
  pdl_wait();
  u32 j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nl_old) {
    up_gen_fill(gen, j - nl_old, offs, adj, dirs);
    return;
  }
  u32 nj = same_l[j];
  if (same_l[j + 1] == nj) return;
  u32 w = offs[nj];
  u32 const e = offs_old[j + 1];
  // FILL_BATCH uses per round, predicated past the row's end (INV marks
  // those: no high entity has that id), so most rows take one round of
  // loads and one of gathers
  for (u32 r = offs_old[j]; r < e; r += FILL_BATCH) {
    u32 a[FILL_BATCH], d[FILL_BATCH];
#pragma unroll
    for (u32 k = 0; k < FILL_BATCH; ++k) {
      a[k] = INV;
      d[k] = 0;
      if (r + k < e) {
        a[k] = adj_old[r + k];
        d[k] = dirs_old[r + k];
      }
    }
#pragma unroll
    for (u32 k = 0; k < FILL_BATCH; ++k) a[k] = a[k] != INV ? newid_h[a[k]] : INV;
#pragma unroll
    for (u32 k = 0; k < FILL_BATCH; ++k)
      if (a[k] != INV) {
        adj[w] = a[k];
        dirs[w] = d[k];
        ++w;
      }
  }
}

// The same fill for long rows (vertex rows, 8 or more uses on average): a
// group of CG lanes (the tuning table's carry_group) walks one
// row, each lane one use, so a row's uses are read and written by
// consecutive lanes; a ballot over the group gives each kept use its place,
// in the old order. (One thread per long row issues loads whose lanes are a
// row apart and fills the load/store queue.) Groups never straddle a warp;
// a group's lanes share their row, so they loop and leave together.
constexpr u32 LONG_ROW_USES = 8;

// the vertex-row fills of a pass's carried pairs share a launch
// (blockIdx.y: the pair)
struct UpFillJob {
  u32 nl_old;
  u32 const* same_l;
  u32 const* newid_h;
  u32 const* offs_old;
  u32 const* adj_old;
  u32 const* dirs_old;
  u32 const* offs;
  u32* adj;
  u32* dirs;
  UpGen gen;
};
struct UpFillJobs {
  UpFillJob j[6];
};

template <u32 CG>
__global__ void k_up_surv_fill_grouped(const __grid_constant__ UpFillJobs jobs)
{
  pdl_wait();
  UpFillJob const& jb = jobs.j[blockIdx.y];
  u32 const nl_old = jb.nl_old;
  u32 const* __restrict__ same_l = jb.same_l;
  u32 const* __restrict__ newid_h = jb.newid_h;
  u32 const* __restrict__ offs_old = jb.offs_old;
  u32 const* __restrict__ adj_old = jb.adj_old;
  u32 const* __restrict__ dirs_old = jb.dirs_old;
  u32 const* __restrict__ offs = jb.offs;
  u32* __restrict__ adj = jb.adj;
  u32* __restrict__ dirs = jb.dirs;
  UpGen const gen = jb.gen;
  u32 const t = blockIdx.x * blockDim.x + threadIdx.x;
  u32 const j = t / CG, g = t % CG;
  if (j >= nl_old) {
    // past the rows' groups (a multiple of CG threads): one thread per
    // generated use
    up_gen_fill(gen, t - nl_old * CG, offs, adj, dirs);
    return;
  }
  u32 const nj = same_l[j];
  if (same_l[j + 1] == nj) return;
  u32 const gbase = (threadIdx.x & 31) & ~(CG - 1);
  u32 const gmask = ((1u << CG) - 1u) << gbase;
  u32 const below = (1u << g) - 1u;
  u32 w = offs[nj];
  u32 const e = offs_old[j + 1];
  for (u32 base = offs_old[j]; base < e; base += CG) {
    u32 const u = base + g;
    u32 na = INV, d = 0;
    if (u < e) {
      na = newid_h[adj_old[u]];
      d = dirs_old[u];
    }
    u32 const kept = (__ballot_sync(gmask, na != INV) & gmask) >> gbase;
    if (na != INV) {
      u32 const pos = w + __popc(kept & below);
      adj[pos] = na;
      dirs[pos] = d;
    }
    w += __popc(kept);
  }
}

// The counts of the carried rows without a gather per use: a surviving row
// keeps its old uses but those of the high entities the pass removed, one
// use in each of their lows' rows, and takes the uses of the entities the
// pass made. k_up_row_lens writes each surviving row's old length (zeroing
// the rows the pass made); k_up_adjust takes a use off for every low of a
// removed high (new id INV) that survives and adds the generated uses.
// (Counting the kept uses row by row gathered a new id for every old use.)
// (the counts of a pass's carried pairs share each launch: blockIdx.y is
// the pair)
struct UpCountJob {
  u32 nl_old, nsame_l, ntail, nh_old, lph, first, nuses;
  u32 const* same_l;
  u32 const* offs_old;
  u32 const* newid_h;
  u32 const* old_loh;
  u32 const* loh;
  u32* cnt;
  u32* surv;
};
struct UpCountJobs {
  UpCountJob j[6];
};

// (grid-stride over a grid of a few blocks per SM: most threads do one or
// two loads, and a block per 256 of them spent the launch scheduling blocks)
__global__ void k_up_row_lens(const __grid_constant__ UpCountJobs jobs)
{
  pdl_wait();
  UpCountJob const& jb = jobs.j[blockIdx.y];
  u32* __restrict__ cnt = jb.cnt;
  u32* __restrict__ surv = jb.surv;
  u32 const end = jb.nl_old + jb.ntail;
  for (u32 j = blockIdx.x * blockDim.x + threadIdx.x; j < end; j += gridDim.x * blockDim.x) {
    if (j >= jb.nl_old) {
      u32 r = jb.nsame_l + (j - jb.nl_old);
      cnt[r] = 0;
      if (surv) surv[r] = 0;
      continue;
    }
    u32 nj = jb.same_l[j];
    if (jb.same_l[j + 1] == nj) continue;
    u32 len = jb.offs_old[j + 1] - jb.offs_old[j];
    cnt[nj] = len;
    if (surv) surv[nj] = len;
  }
}

__global__ void k_up_adjust(const __grid_constant__ UpCountJobs jobs)
{
  pdl_wait();
  UpCountJob const& jb = jobs.j[blockIdx.y];
  u64 const end = (u64)jb.nh_old + (jb.nuses > jb.first ? jb.nuses - jb.first : 0u);
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < end;
       t += (u64)gridDim.x * blockDim.x) {
    if (t < jb.nh_old) {
      if (jb.newid_h[t] != INV) continue;
      for (u32 k = 0; k < jb.lph; ++k) {
        u32 l = jb.old_loh[(size_t)t * jb.lph + k];
        u32 nl = jb.same_l[l];
        if (jb.same_l[l + 1] == nl) continue;
        atomicSub(&jb.cnt[nl], 1u);
        if (jb.surv) atomicSub(&jb.surv[nl], 1u);
      }
      continue;
    }
    u32 u = jb.first + (u32)(t - jb.nh_old);
    atomicAdd(&jb.cnt[jb.loh[u]], 1u);
  }
}

u32* carry_new_ids(u32 const* same, u32 n, cudaStream_t s)
{
  u32* newid = dalloc<u32>(n ? n : 1, s);
  if (n) {
    CK(launch_kernel(k_new_ids, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, same, newid));
    CK_LAUNCH();
  }
  return newid;
}

namespace {

// one carried upward adjacency between its count and its fill (the counts
// of every carried pair are scanned together in one launch)
struct UpCarry {
  u32 low = 0, high = 0;
  u32 nl_old = 0, nl = 0, nsame_l = 0, nh_old = 0, nuses = 0, nuses_old = 0, first = 0, lph = 0;
  bool long_rows = false;
  u32 const* same_l = nullptr;
  u32 const* newid_h = nullptr;
  u32 const* loh = nullptr;
  u32* cnt = nullptr;
  u32* surv = nullptr;
  UpAdj u;
  UpCountJob cj;
};

// the pair's arrays and its count job: false when the pair is not carried
bool carry_up_setup(Mesh& m, Mesh& out, u32 low, u32 high, u32 const* same_l, u32 nsame_l,
    u32 nsame_h, u32 const* newid_h, UpCarry& c)
{
  if (!m.have_up[low][high] || out.have_up[low][high]) return false;
  if (!out.has_dim(high) || !out.has_dim(low)) return false;
  if (low > 0 && !out.down[high][low]) return false;  // its search is not worth it here
  cudaStream_t s = out.s;
  c.low = low;
  c.high = high;
  c.nl_old = m.counts[low];
  c.nl = out.count(low);
  u32 nh = out.count(high);
  if (nsame_l > c.nl || nsame_l > c.nl_old) throw Failure(E_ARG, "carry_up: survivor count");
  c.nsame_l = nsame_l;
  c.same_l = same_l;
  c.newid_h = newid_h;
  c.lph = deg(high, low);
  c.nuses = nh * c.lph;
  c.first = nsame_h * c.lph;
  c.loh = out.ask_down(high, low);
  UpAdj const& old = m.up[low][high];
  c.nh_old = m.counts[high];
  // cnt: kept + generated uses per new row; surv (kept only when the old
  // rows were sorted): each row's count of leading uses, in order
  c.cnt = dalloc<u32>((size_t)c.nl + 1, s);
  c.surv = m.up_sorted[low][high] ? dalloc<u32>((size_t)c.nl + 1, s) : nullptr;
  c.nuses_old = m.counts[high] * c.lph;
  // rows of 8 or more uses on average (vertex rows) take a lane group each
  c.long_rows = c.nl_old && (u64)c.nuses_old >= (u64)LONG_ROW_USES * c.nl_old;
  // the count kernels' job (launched with the other pairs')
  UpCountJob& j = c.cj;
  j.nl_old = c.nl_old;
  j.nsame_l = nsame_l;
  j.ntail = c.nl + 1 - nsame_l;
  j.nh_old = c.nh_old;
  j.lph = c.lph;
  j.first = c.first;
  j.nuses = c.nuses;
  j.same_l = same_l;
  j.offs_old = old.offs;
  j.newid_h = newid_h;
  j.old_loh = m.ask_down(high, low);
  j.loh = c.loh;
  j.cnt = c.cnt;
  j.surv = c.surv;
  c.u.offs = dalloc<u32>((size_t)c.nl + 1, s);
  return true;
}

// after the scan of the counts: the rows' fill (edge and face rows here, a
// launch per pair; vertex rows into `grouped`, launched for all pairs
// together), and the adjacency installed
void carry_up_fill(Mesh& m, Mesh& out, UpCarry& c, UpFillJobs& grouped, u32& ngrouped,
    u64& gmost, double& gbytes)
{
  cudaStream_t s = out.s;
  UpAdj const& old = m.up[c.low][c.high];
  UpAdj& u = c.u;
  u.adj = dalloc<u32>(c.nuses, s);
  u.dirs = dalloc<u32>(c.nuses, s);
  u32 const cg = tuned(TK_CARRY_GROUP), gb = tuned(TK_GATHER_BLOCK);
  u64 const ngen = c.nuses > c.first ? c.nuses - c.first : 0;
  UpGen const gen{c.first, c.nuses, c.lph, c.loh, c.cnt};
  if (c.long_rows) {
    grouped.j[ngrouped++] = UpFillJob{c.nl_old, c.same_l, c.newid_h, old.offs, old.adj,
        old.dirs, u.offs, u.adj, u.dirs, gen};
    gmost = std::max<u64>(gmost, (u64)c.nl_old * cg + ngen);
    gbytes += 8.0 * (c.nl_old + 1) + 8.0 * c.nuses_old + 4.0 * c.nh_old + 4.0 * (c.nl + 1) +
        8.0 * c.first + 20.0 * ngen;
  } else if (c.nl_old || ngen) {
    // each array once: same_l and the old offsets, the old rows' highs and
    // directions, the highs' new ids, the new offsets, the kept uses (first)
    // written as highs and directions; per generated use its low, the
    // row's offset and count, and the use written
    // (the fill of edge and face rows, the largest single kernel of an
    // adapt, is probed on its own: carry_up_fill)
    PROBE(P_CARRY_UP_FILL, s, 8.0 * (c.nl_old + 1) + 8.0 * c.nuses_old + 4.0 * c.nh_old +
        4.0 * (c.nl + 1) + 8.0 * c.first + 20.0 * ngen);
    CK(launch_kernel(k_up_surv_fill, dim3(grid_for((u64)c.nl_old + ngen, gb)), dim3(gb), 0,
        s, c.nl_old, c.same_l, c.newid_h, old.offs, old.adj, old.dirs, u.offs, u.adj, u.dirs,
        gen));
    CK_LAUNCH();
  }
}

// after every fill: the counts freed and the adjacency installed
void carry_up_install(Mesh& out, UpCarry& c)
{
  cudaStream_t s = out.s;
  UpAdj& u = c.u;
  dev_free(c.cnt, s);
  if (c.surv) {
    u.pre = c.surv;
    u.npre = c.first;
  }
  out.up[c.low][c.high] = u;
  out.have_up[c.low][c.high] = true;
  out.up_sorted[c.low][c.high] = false;
}

}  // namespace

void carry_up_all(Mesh& m, Mesh& out, u32* const* same_of, u32 const* nsame_of,
    u32* const* newid_of)
{
  cudaStream_t s = out.s;
  UpCarry cs[6];
  u32 nc = 0;
  // each old high entity's new id (INV when it did not survive): from the
  // survivors' scan where it wrote them, else computed here, once per
  // high dimension
  u32* own_newid[4] = {nullptr, nullptr, nullptr, nullptr};
  for (u32 h = 1; h <= m.dim; ++h)
    for (u32 l = 0; l < h; ++l) {
      if (!same_of[h] || !same_of[l]) continue;
      if (!m.have_up[l][h] || out.have_up[l][h]) continue;
      u32 const* newid_h = newid_of[h];
      if (!newid_h) {
        if (!own_newid[h]) own_newid[h] = carry_new_ids(same_of[h], m.counts[h], s);
        newid_h = own_newid[h];
      }
      if (carry_up_setup(m, out, l, h, same_of[l], nsame_of[l], nsame_of[h], newid_h, cs[nc]))
        ++nc;
    }
  if (nc) {
    // every pair's counts in one launch per stage: the surviving rows'
    // lengths, then the removed and generated uses
    UpCountJobs cj;
    u64 most_rows = 0, most_adj = 0;
    double bytes_rows = 0, bytes_adj = 0;
    for (u32 k = 0; k < nc; ++k) {
      UpCarry const& c = cs[k];
      cj.j[k] = c.cj;
      u64 const ngen = c.nuses > c.first ? c.nuses - c.first : 0;
      most_rows = std::max<u64>(most_rows, (u64)c.nl_old + c.cj.ntail);
      most_adj = std::max<u64>(most_adj, (u64)c.nh_old + ngen);
      // same_l and the old offsets, the new counts (and kept counts); the
      // highs' new ids, and per generated use its low and the count
      bytes_rows += 8.0 * (c.nl_old + 1) + 4.0 * c.nl * (c.surv ? 2.0 : 1.0);
      bytes_adj += 4.0 * c.nh_old + 8.0 * ngen;
    }
    u32 const gb = tuned(TK_GATHER_BLOCK);
    {
      PROBE(P_CARRY_UP, s, bytes_rows);
      CK(launch_kernel(k_up_row_lens, dim3(std::min<u32>(grid_for(most_rows, gb),
          148u * 8u * 256u / gb), nc), dim3(gb), 0, s, cj));
      CK_LAUNCH();
    }
    {
      PROBE(P_UP_COUNT, s, bytes_adj);
      CK(launch_kernel(k_up_adjust, dim3(std::min<u32>(grid_for(most_adj, gb),
          148u * 8u * 256u / gb), nc), dim3(gb), 0, s, cj));
      CK_LAUNCH();
    }
  }
  ScanJob jobs[6];
  for (u32 k = 0; k < nc; ++k) jobs[k] = ScanJob{cs[k].cnt, cs[k].u.offs, nullptr, nullptr,
      cs[k].nl, 0};
  exscan_jobs(jobs, nc, s);
  UpFillJobs grouped;
  u32 ngrouped = 0;
  u64 gmost = 0;
  double gbytes = 0;
  for (u32 k = 0; k < nc; ++k) carry_up_fill(m, out, cs[k], grouped, ngrouped, gmost, gbytes);
  if (ngrouped) {
    PROBE(P_CARRY_UP, s, gbytes);
    u32 const cg = tuned(TK_CARRY_GROUP), gb = tuned(TK_GATHER_BLOCK);
    auto kf = cg == 4 ? k_up_surv_fill_grouped<4>
            : cg == 16 ? k_up_surv_fill_grouped<16> : k_up_surv_fill_grouped<8>;
    CK(launch_kernel(kf, dim3(grid_for(gmost, gb), ngrouped), dim3(gb), 0, s, grouped));
    CK_LAUNCH();
  }
  for (u32 k = 0; k < nc; ++k) carry_up_install(out, cs[k]);
  for (u32 h = 0; h < 4; ++h) dev_free(own_newid[h], s);
}

u32 const* Mesh::ask_down(u32 high, u32 low)
{
  if (down[high][low]) return down[high][low];
  if (low == high) {
    u32 n = counts[high];
    u32* a = dalloc<u32>(n, s);
    iota_u32(a, n, 1, s);
    down[high][low] = a;
  } else if (low > 0) {
    u32 nh = count(high);
    u32* out = dalloc<u32>((size_t)nh * deg(high, low), s);
    reflect_range(high, low, 0, out);
    down[high][low] = out;
  } else if (high == 1 && dim == 3) {
    // edges in 3D bridge the vertex star (mesh.cpp:160-168)
    Graph const& vv = ask_star(0, dim);
    u32 nv = counts[0];
    u32* degree = dalloc<u32>(nv, s);
    if (nv) {
      CK(launch_kernel(k_bridge_degree, dim3(grid_for(nv)), dim3(BLOCK), 0, s, nv, vv.offs, 0, vv.adj, degree));
      CK_LAUNCH();
    }
    u32* bo = exscan_new(degree, nv, s);
    dev_free(degree, s);
    u32 ne = read_u32(bo + nv, s);
    u32* voe = dalloc<u32>((size_t)ne * 2, s);
    if (nv) {
      CK(launch_kernel(k_bridge_edges, dim3(grid_for(nv)), dim3(BLOCK), 0, s, nv, vv.offs, vv.adj, bo, voe));
      CK_LAUNCH();
    }
    dev_free(bo, s);
    set_ents(1, ne, voe);
  } else {
    // sides from the element dual (mesh.cpp:169-179)
    u32 const* du = ask_dual();
    u32 nel = counts[dim];
    u32 spe = deg(dim, dim - 1);
    u32* degree = dalloc<u32>(nel, s);
    if (nel) {
      CK(launch_kernel(k_bridge_degree, dim3(grid_for(nel)), dim3(BLOCK), 0, s, nel, nullptr, spe, du, degree));
      CK_LAUNCH();
    }
    u32* bo = exscan_new(degree, nel, s);
    dev_free(degree, s);
    u32 ns = read_u32(bo + nel, s);
    u32 vps = deg(dim - 1, 0);
    u32* vos = dalloc<u32>((size_t)ns * vps, s);
    if (nel) {
      CK(launch_kernel(k_derive_sides, dim3(grid_for(nel)), dim3(BLOCK), 0, s, dim, nel, du, bo, down[dim][0], vos));
      CK_LAUNCH();
    }
    dev_free(bo, s);
    set_ents(dim - 1, ns, vos);
  }
  return down[high][low];
}

UpAdj const& Mesh::ask_up(u32 low, u32 high, bool sorted)
{
  if (have_up[low][high]) {
    if (sorted && !up_sorted[low][high]) {
      sort_up_rows(high, low, counts[high], counts[low], up[low][high], s);
      up_sorted[low][high] = true;
      dev_free(up[low][high].pre, s);
      up[low][high].pre = nullptr;
      up[low][high].npre = 0;
    }
    return up[low][high];
  }
  if (low == high) {
    u32 n = counts[high];
    UpAdj u;
    u.offs = dalloc<u32>((size_t)n + 1, s);
    iota_u32(u.offs, n + 1, 1, s);
    u.adj = dalloc<u32>(n, s);
    iota_u32(u.adj, n, 1, s);
    u.dirs = dalloc<u32>(n, s);
    fill_u32(u.dirs, n, 0, s);
    up[low][high] = u;
    up_sorted[low][high] = true;
  } else {
    u32 const* loh = ask_down(high, low);
    if (sorted) {
      up_from_down(high, low, counts[high], counts[low], loh, up[low][high], s);
      up_sorted[low][high] = true;
    } else {
      up_from_down_unsorted(high, low, counts[high], counts[low], loh, up[low][high], s);
      up_sorted[low][high] = false;
    }
  }
  have_up[low][high] = true;
  return up[low][high];
}

Graph const& Mesh::ask_star(u32 low, u32 high)
{
  if (have_star[low][high]) return star[low][high];
  Graph g;
  if (low == high) {
    u32 n = counts[low];
    g.offs = dalloc<u32>((size_t)n + 1, s);
    fill_u32(g.offs, n + 1, 0, s);
    g.adj = dalloc<u32>(1, s);
  } else if (low == 0 && high == dim && dim != 1 && has_dim(1)) {
    Graph const& vv = ask_star(0, 1);
    u32 n = counts[0];
    g.offs = dalloc<u32>((size_t)n + 1, s);
    CK(cudaMemcpyAsync(g.offs, vv.offs, sizeof(u32) * (n + 1), cudaMemcpyDeviceToDevice, s));
    g.nadj = vv.nadj;
    g.adj = dalloc<u32>(g.nadj, s);
    CK(cudaMemcpyAsync(g.adj, vv.adj, sizeof(u32) * g.nadj, cudaMemcpyDeviceToDevice, s));
  } else if (low == 0 && high == 1) {
    // get_vertex_edge_star (star.cpp:135-160)
    u32 n = count(0);
    u32 const* voe = ask_down(1, 0);
    UpAdj const& ev = ask_up(0, 1);
    g.nadj = counts[1] * 2;
    g.offs = dalloc<u32>((size_t)n + 1, s);
    CK(cudaMemcpyAsync(g.offs, ev.offs, sizeof(u32) * (n + 1), cudaMemcpyDeviceToDevice, s));
    g.adj = dalloc<u32>(g.nadj, s);
    if (g.nadj) {
      CK(launch_kernel(k_vertex_edge_star, dim3(grid_for(g.nadj)), dim3(BLOCK), 0, s, g.nadj, ev.adj, ev.dirs, voe, g.adj));
      CK_LAUNCH();
    }
  } else if (low == 1 && high == 2) {
    // get_edge_triangle_star (star.cpp:189-218)
    u32 n = count(1);
    u32 const* eot = ask_down(2, 1);
    UpAdj const& te = ask_up(1, 2);
    u32 nuse = counts[2] * 3;
    g.nadj = nuse * 2;
    g.offs = dalloc<u32>((size_t)n + 1, s);
    CK(launch_kernel(k_scale_offsets, dim3(grid_for(n + 1)), dim3(BLOCK), 0, s, te.offs, n + 1, 2, g.offs));
    CK_LAUNCH();
    g.adj = dalloc<u32>(g.nadj, s);
    if (nuse) {
      CK(launch_kernel(k_edge_tri_star, dim3(grid_for(nuse)), dim3(BLOCK), 0, s, nuse, te.adj, te.dirs, eot, g.adj));
      CK_LAUNCH();
    }
  } else if (low == 1 && high == 3 && has_dim(2)) {
    // get_edge_tet_star (star.cpp:255-293)
    Graph const& ts = ask_star(1, 2);
    u32 n = count(1);
    u32 const* eor = ask_down(3, 1);
    UpAdj const& re = ask_up(1, 3);
    u32* degree = dalloc<u32>(n, s);
    if (n) {
      CK(launch_kernel(k_sum_degrees, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, ts.offs, re.offs, degree));
      CK_LAUNCH();
    }
    g.offs = exscan_new(degree, n, s);
    dev_free(degree, s);
    g.nadj = ts.nadj + counts[3] * 6;
    g.adj = dalloc<u32>(g.nadj, s);
    if (n) {
      CK(launch_kernel(k_edge_tet_star, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, g.offs, ts.offs, ts.adj, re.offs,
          re.adj, re.dirs, eor, g.adj));
      CK_LAUNCH();
    }
  } else {
    // get_star_general (star.cpp:14-111)
    u32 n = count(low);
    UpAdj const& hl = ask_up(low, high);
    u32 const* loh = ask_down(high, low);
    u32 lph = deg(high, low);
    u32* degree = dalloc<u32>(n, s);
    u32* err = mb->dev + 60;
    CK(cudaMemsetAsync(err, 0, sizeof(u32), s));
    if (n) {
      CK(launch_kernel(k_star_general, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, hl.offs, hl.adj, loh, lph,
          nullptr, degree, nullptr, err));
      CK_LAUNCH();
    }
    g.offs = exscan_new(degree, n, s);
    dev_free(degree, s);
    g.nadj = read_u32(g.offs + n, s);
    g.adj = dalloc<u32>(g.nadj, s);
    if (n) {
      CK(launch_kernel(k_star_general, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, hl.offs, hl.adj, loh, lph, g.offs,
          nullptr, g.adj, err));
      CK_LAUNCH();
    }
    if (read_u32(err, s)) throw Failure(E_ARG, "star wider than 256 entries");
  }
  star[low][high] = g;
  have_star[low][high] = true;
  return star[low][high];
}

u32 const* Mesh::ask_dual()
{
  if (dual) return dual;
  u32 nel = count(dim), spe = deg(dim, dim - 1);
  u32* out = dalloc<u32>((size_t)nel * spe, s);
  if (has_dim(dim - 1)) {
    u32 const* soe = ask_down(dim, dim - 1);
    UpAdj const& es = ask_up(dim - 1, dim, false);
    if (nel) {
      CK(launch_kernel(k_dual_from_sides, dim3(grid_for(nel)), dim3(BLOCK), 0, s, nel, spe, soe, es.offs, es.adj, out));
      CK_LAUNCH();
    }
  } else {
    u32 const* voe = ask_down(dim, 0);
    UpAdj const& ev = ask_up(0, dim);
    u32* err = mb->dev + 61;
    CK(cudaMemsetAsync(err, 0, sizeof(u32), s));
    if (nel) {
      CK(launch_kernel(k_dual_from_verts, dim3(grid_for((u64)nel * spe)), dim3(BLOCK), 0, s, dim, nel, voe, ev.offs,
          ev.adj, out, err));
      CK_LAUNCH();
    }
    if (read_u32(err, s)) throw Failure(E_ARG, "vertex with more than 256 elements");
  }
  dual = out;
  return dual;
}

// ---------------------------------------------------------------------------
// geometry: qualities, sizes, edge lengths (quality.cpp, size.cpp)


__global__ void k_elem_quality(u32 dim, u32 ne, u32 const* __restrict__ voe,
    double const* __restrict__ x, double* __restrict__ q,
    unsigned long long* minkey)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  double qi = DBL_MAX;
  if (i < ne) {
    u32 vpe = deg(dim, 0);
    double ex[4][3];
    for (u32 j = 0; j < vpe; ++j) load3(x, voe[(size_t)i * vpe + j], ex[j]);
    qi = dim >= 2 ? elem_quality(dim, ex, 1) : 1.0;
    q[i] = qi;
  }
  // min over elements below DBL_MAX, as doubles_min's `a[i] < min` keeps
  unsigned long long key = (qi < DBL_MAX) ? order_key(qi) : ~0ull;
  for (int o = 16; o; o >>= 1) {
    unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
    key = other < key ? other : key;
  }
  if ((threadIdx.x & 31) == 0 && key != ~0ull) atomicMin(minkey, key);
}

// The cache holds ne qualities followed by one 8-byte slot with the
// order-preserving key of their minimum.
double const* Mesh::qualities()
{
  if (qual_cache) return qual_cache;
  u32 ne = count(dim);
  qual_cache = dalloc<double>((size_t)ne + 1, s);
  unsigned long long* mk = reinterpret_cast<unsigned long long*>(qual_cache + ne);
  CK(cudaMemsetAsync(mk, 0xff, sizeof(unsigned long long), s));
  if (ne) {
    PROBE(P_ELEM_QUALITY, s, 4.0 * deg(dim, 0) * ne + 24.0 * counts[0] + 8.0 * ne);
    u32 const qb = tuned(TK_QUALITY_BLOCK);
    CK(launch_kernel(k_elem_quality, dim3(grid_for(ne, qb)), dim3(qb), 0, s, dim, ne,
        ask_down(dim, 0), coords(), qual_cache, mk));
    CK_LAUNCH();
  }
  return qual_cache;
}

// mesh_min_quality (quality.cpp:67-73) over every element
double Mesh::min_quality()
{
  double const* q = qualities();
  u32 ne = count(dim);
  u32 const* w = mb->read(s, reinterpret_cast<u32 const*>(q + ne), 2);
  unsigned long long k = (unsigned long long)w[0] | ((unsigned long long)w[1] << 32);
  if (k == ~0ull) return DBL_MAX;
  return from_order_key(k);
}

__global__ void k_elem_size(u32 dim, u32 ne, u32 const* __restrict__ voe,
    double const* __restrict__ x, double* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  u32 vpe = deg(dim, 0);
  double ex[4][3];
  for (u32 j = 0; j < vpe; ++j) load3(x, voe[(size_t)i * vpe + j], ex[j]);
  double v;
  if (dim == 3)
    v = tet_volume(ex);
  else if (dim == 2)
    v = tri_area(ex[0], ex[1], ex[2]);
  else
    v = sqrt(sqdist3(ex[1], ex[0]));
  out[i] = v;
}

double* Mesh::element_sizes()
{
  u32 ne = count(dim);
  double* out = dalloc<double>(ne, s);
  if (ne) {
    CK(launch_kernel(k_elem_size, dim3(grid_for(ne)), dim3(BLOCK), 0, s, dim, ne, ask_down(dim, 0), coords(), out));
    CK_LAUNCH();
  }
  return out;
}

__global__ void k_measure_edges(u32 ne, u32 const* __restrict__ voe,
    double const* __restrict__ x, double const* __restrict__ h, double* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  u32 a = voe[i * 2], b = voe[i * 2 + 1];
  double xa[3], xb[3];
  load3(x, a, xa);
  load3(x, b, xb);
  double len = sqrt(sqdist3(xb, xa));
  double want = (h[a] + h[b]) / 2;
  out[i] = len / want;
}

double* Mesh::measure_edges()
{
  u32 ne = count(1);
  Tag* t = find_tag(0, "adapt_size");
  if (!t) throw Failure(E_ARG, "mesh has no adapt_size vertex field");
  double* out = dalloc<double>(ne, s);
  if (ne) {
    CK(launch_kernel(k_measure_edges, dim3(grid_for(ne)), dim3(BLOCK), 0, s, ne, ask_down(1, 0), coords(),
        static_cast<double const*>(t->data), out));
    CK_LAUNCH();
  }
  return out;
}

}  // namespace osh
