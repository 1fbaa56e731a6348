// Luby-style maximal independent set with goodness priority (indset.cpp) and
// the small shared kernels of the passes: marking, class inheritance,
// expansion, global renumbering.
//
// The star graph is never materialised for the independent set: an edge's
// neighbours are the other edges of the tets around it (up(1,3) then
// down(3,1)), a vertex's neighbours the far ends of its edges (up(0,1)).
// That is exactly the neighbour set of the reference's star(1,3) /
// star(0,1) (star.cpp:135-293); the selection rule depends only on that set.
#include <algorithm>
#include <atomic>
#include <vector>

#include "passes.hpp"

namespace osh {

PassStats& last_pass_stats()
{
  static thread_local PassStats s;
  return s;
}

// control words of the single-launch rounds (mailbox slots 44-50)
constexpr u32 COOP_CTL_SLOT = 44, COOP_CTL_WORDS = 7;
// (what the rounds read back: the words below; the control words' layout
// is given at k_indset_coop)
static_assert(COOP_CTL_SLOT + COOP_CTL_WORDS == INDSET_FETCH_SLOTS, "mailbox slots");

// also zeroes the control words of the rounds
// neighbourhood walks: mode 0 = vertices via edges, mode 1 = edges via
// elements (3D tets or 2D triangles)
struct Nbrs {
  u32 mode;
  u32 const* offs;   // up(ent, via)
  u32 const* adj;
  u32 const* dirs;
  u32 const* down;   // down(via, ent) or verts_of_edges
  u32 per;           // entities per via-entity
};

// indset_at_vert (indset.cpp:55-84) for entity i: out of the set if a
// neighbour is in it; in the set if no undecided neighbour beats it (higher
// goodness, or equal goodness and a lower global id); undecided otherwise.
// The rounds here update one state array in place and keep a list of the
// entities still undecided, so a round's work is the undecided entities,
// not all of them. The set is the same as the reference's synchronous
// rounds give: states only ever change from undecided to decided, so a
// state read during a round is either the one of the round before or the
// final one, and an entity that joins sees every better neighbour decided
// out -- the lexicographically first independent set in goodness order,
// whatever the timing. (A state read from the round before only delays a
// decision to a later round.)
//
// A group of G lanes (G divides 32, so a group never straddles a warp)
// walks the entity's upward entries l, l + G, ...; each lane folds its
// neighbours into two flags, and two ballots over the group combine them.
// (One thread per long row issues loads whose lanes are a row apart and
// fills the load/store queue.)
//
// All rounds run in one launch: a cooperative grid (every block resident)
// sets the states and lists the candidates, then runs round 0 over them and
// later rounds over the list the round before left, separated by a grid
// barrier (by a block barrier when block 0 alone takes few candidates),
// until a round leaves no entity undecided or 100 rounds have run.
// Control words (zero on entry but [1]: see the prologue): [0] barrier
// arrivals, [1] barrier generation (only its changes count), [2..4]
// length of the list round r builds for round r + 1, r + 1 = 0, 1, 2 mod 3
// (round r zeroes the counter of round r + 2, last read after the barrier
// of round r - 2 that every block has passed), [5] rounds run, [6] a barrier
// wait gave up. States and list entries are read past L1 (L1 may keep a
// line another block has since rewritten; a stale undecided state would
// only delay the decision, but a line kept stale for good would never let
// it end, and a stale list entry would name the wrong entity). The
// barrier's wait is bounded: after COOP_SPIN_LIMIT polls it sets [6] and
// every block leaves.
constexpr u32 COOP_SPIN_LIMIT = 1u << 24;

__device__ inline bool coop_barrier(u32* ctl)
{
  __syncthreads();
  if (threadIdx.x == 0) {
    u32 const g0 = *(volatile u32*)&ctl[1];
    __threadfence();
    if (atomicAdd(&ctl[0], 1u) + 1u == gridDim.x) {
      *(volatile u32*)&ctl[0] = 0;
      __threadfence();
      atomicAdd(&ctl[1], 1u);
    } else {
      u32 spins = 0;
      while (*(volatile u32*)&ctl[1] == g0) {
        if (++spins > COOP_SPIN_LIMIT) {
          atomicOr(&ctl[6], 1u);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile u32*)&ctl[6] == 0;
}

// (at least 4 blocks per SM: without a minimum the compiler held the
// kernel to 32 registers and spilled)
template <int G>
__global__ void __launch_bounds__(BLOCK, 4) k_indset_coop(u32 n, Nbrs g,
    u32 const* __restrict__ filter, u32* st, u32* wl0, u32* wl1,
    double const* __restrict__ good, u64 const* __restrict__ glob, u32* ctl)
{
  pdl_wait();
  u32 const lg = threadIdx.x % G;
  u32 const gbase = (threadIdx.x & 31) & ~(u32)(G - 1);
  u32 const gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << gbase;
  u32 const lane = threadIdx.x & 31;
  u32 const stride = gridDim.x * blockDim.x;
  // The states (the filter's candidates undecided, the rest out of the set)
  // and round 0's list, the candidates, appended a warp at a time to the
  // list whose length is control word 2 (zero on entry: this kernel zeroes
  // the list lengths when it settles, the host when a set fails); then the
  // grid barrier, so round 0 sees every state and the whole list
  for (u64 b = (u64)blockIdx.x * blockDim.x; b < n; b += stride) {
    u32 const i = (u32)b + threadIdx.x;
    bool const c = i < n && (!filter || filter[i]);
    if (i < n) __stcg(&st[i], c ? (u32)UNKNOWN : (u32)NOT_IN_SET);
    unsigned const want = __ballot_sync(0xffffffffu, c);
    if (want) {
      u32 const leader = __ffs(want) - 1;
      u32 base = 0;
      if (lane == leader) base = atomicAdd(&ctl[2], (u32)__popc(want));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (c) wl1[base + __popc(want & ((1u << lane) - 1u))] = i;
    }
  }
  __threadfence();
  if (!coop_barrier(ctl)) return;
  // A short candidate list (two sweeps of one block at most) is left to
  // block 0, whose rounds are separated by block barriers instead of grid
  // barriers. Every block decides the same: one reading the length after
  // block 0 has gone on reads a later list's length or zero, never more.
  bool const solo = (u64)(*(volatile u32*)&ctl[2]) * G <= 2u * blockDim.x;
  if (solo && blockIdx.x != 0) return;
  u32 const rstride = solo ? blockDim.x : stride;
  for (u32 r = 0; r < MAX_INDSET_ROUNDS; ++r) {
    // round 0 walks the candidates, round r > 0 the list round r - 1 left
    u32 const len = *(volatile u32*)&ctl[2 + r % 3];
    u32 const* list = (r % 2 == 1) ? wl0 : wl1;
    u32* next = (r % 2 == 0) ? wl0 : wl1;
    u32* next_len = &ctl[2 + (r + 1) % 3];
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl[2 + (r + 2) % 3] = 0;
    for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < (u64)len * G; t += rstride) {
      // past L1, like the states: the lists alternate between two
      // buffers, so this block may hold lines of this one from two rounds
      // ago that other blocks have since rewritten
      u32 const i = __ldcg(&list[t / G]);
      u32 const s0 = __ldcg(&st[i]);
      bool undecided = false;
      if (s0 == UNKNOWN) {
        u32 const rb = g.offs[i], re = g.offs[i + 1];
        double const myg = good[i];
        u64 const myid = glob ? glob[i] : (u64)i;
        bool in_set = false, beaten = false;
        auto visit = [&](u32 o) {
          u32 so = __ldcg(&st[o]);
          if (so == IN_SET) in_set = true;
          if (so == NOT_IN_SET) return;
          double og = good[o];
          u64 oid = glob ? glob[o] : (u64)o;
          if ((myg == og && oid < myid) || myg < og) beaten = true;
        };
        for (u32 j = rb + lg; j < re; j += G) {
          if (g.mode == 0) {
            visit(g.down[g.adj[j] * 2 + (1 - g.dirs[j])]);
          } else {
            u32 const* ds = g.down + (size_t)g.adj[j] * g.per;
            for (u32 k = 0; k < g.per; ++k)
              if (ds[k] != i) visit(ds[k]);
          }
        }
        bool const any_in = (__ballot_sync(gmask, in_set) & gmask) != 0;
        bool const lost = (__ballot_sync(gmask, beaten) & gmask) != 0;
        if (lg == 0) {
          if (any_in)
            __stcg(&st[i], (u32)NOT_IN_SET);
          else if (!lost)
            __stcg(&st[i], (u32)IN_SET);
          else
            undecided = true;
        }
      }
      // the undecided entities of this pass of the loop, appended to the
      // next list: one counter update per warp
      unsigned const act = __activemask();
      unsigned const want = __ballot_sync(act, undecided);
      if (want) {
        u32 const leader = __ffs(want) - 1;
        u32 base = 0;
        if (lane == leader) base = atomicAdd(next_len, (u32)__popc(want));
        base = __shfl_sync(act, base, leader);
        if (undecided) next[base + __popc(want & ((1u << lane) - 1u))] = i;
      }
    }
    __threadfence();
    if (solo)
      __syncthreads();
    else if (!coop_barrier(ctl))
      return;
    if (*(volatile u32*)next_len == 0) {
      // settled: every block still running has passed the last barrier and
      // reads only next_len (zero) from here, so the list lengths go back to
      // zero for the next set's prologue
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl[5] = r + 1;
        ctl[2] = ctl[3] = ctl[4] = 0;
      }
      return;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl[5] = MAX_INDSET_ROUNDS;
}

namespace {
// blocks of BLOCK threads a cooperative launch uses on this device: the
// tuning table's indset_blocks per SM, at most as many as are resident
template <int G>
u32 coop_blocks()
{
  static std::atomic<u32> per_sm_of[64];
  static std::atomic<u32> sms_of[64];
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return 0;
  if (!sms_of[dev].load()) {
    int per_sm = 0, sms = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_indset_coop<G>, BLOCK, 0));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    per_sm_of[dev].store((u32)per_sm);
    sms_of[dev].store((u32)sms);
  }
  u32 per_sm = per_sm_of[dev].load(), want = tuned(TK_INDSET_BLOCKS);
  if (want && want < per_sm) per_sm = want;
  return per_sm * sms_of[dev].load();
}

template <int G>
void launch_coop(u32 n, Nbrs const& g, u32 const* filter, u32* st, u32* wl,
    double const* good, u64 const* glob, u32* ctl, cudaStream_t s)
{
  u32 blocks = std::min<u32>(grid_for((u64)n * G), coop_blocks<G>());
  if (!blocks) throw Failure(E_CUDA, "independent set: no resident blocks");
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(BLOCK);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelEx(&cfg, k_indset_coop<G>, n, g, filter, st, wl, wl + n, good, glob,
      ctl));
  CK_LAUNCH();
}
}  // namespace

// number of upward uses walked per round (edges of vertices / elements of
// edges), for the probe's byte count
static u32 read_cached_uses(Mesh& m, u32 ent_dim)
{
  return ent_dim == 0 ? 2u * m.counts[1] : deg(m.dim, 1) * m.counts[m.dim];
}

u32* find_indset(Mesh& m, u32 ent_dim, u32 const* filter, double const* good, bool check)
{
  u32 n = m.count(ent_dim);
  Nbrs g{};
  if (ent_dim == 0) {
    UpAdj const& u = m.ask_up(0, 1, false);
    g.mode = 0;
    g.offs = u.offs;
    g.adj = u.adj;
    g.dirs = u.dirs;
    g.down = m.ask_down(1, 0);
    g.per = 2;
  } else if (ent_dim == 1 && m.dim >= 2) {
    UpAdj const& u = m.ask_up(1, m.dim, false);
    g.mode = 1;
    g.offs = u.offs;
    g.adj = u.adj;
    g.dirs = u.dirs;
    g.down = m.ask_down(m.dim, 1);
    g.per = deg(m.dim, 1);
  } else {
    throw Failure(E_ARG, "independent sets are built on vertices or edges");
  }
  // global numbers held as the identity flag are the local index, which is
  // what the kernel compares when it has no array
  u64 const* glob = m.parallel ? m.globals[ent_dim] : nullptr;
  u32* a = dalloc<u32>(n, m.s);
  u32* b = dalloc<u32>(2 * (size_t)n, m.s);  // the two lists of undecided entities
  // One cooperative launch sets the states, lists the candidates and runs
  // every round, updating a in place; its control words (mailbox slots
  // COOP_CTL_SLOT..) come back with slots 1-3, which a caller that left
  // flags there reads after this call without a read-back of its own. With
  // no entity, only the rounds count is zeroed.
  u32* ctl = m.mb->dev + COOP_CTL_SLOT;
  if (n) {
    double nuse = (double)read_cached_uses(m, ent_dim);
    double avg_row = nuse / n;
    u32 lanes = avg_row >= 8.0 ? tuned(TK_INDSET_VERT_GROUP)
              : avg_row >= 3.0 ? tuned(TK_INDSET_EDGE_GROUP) : 1u;
    if (lanes == 16) launch_coop<16>(n, g, filter, a, b, good, glob, ctl, m.s);
    else if (lanes == 8) launch_coop<8>(n, g, filter, a, b, good, glob, ctl, m.s);
    else if (lanes == 4) launch_coop<4>(n, g, filter, a, b, good, glob, ctl, m.s);
    else if (lanes == 2) launch_coop<2>(n, g, filter, a, b, good, glob, ctl, m.s);
    else launch_coop<1>(n, g, filter, a, b, good, glob, ctl, m.s);
  } else {
    CK(cudaMemsetAsync(ctl + 5, 0, sizeof(u32), m.s));
  }
  dev_free(b, m.s);
  if (check) {
    m.mb->fetch(m.s, INDSET_FETCH_SLOTS);
    try {
      indset_check(m);
    } catch (...) {
      dev_free(a, m.s);
      throw;
    }
  }
  return a;
}

void indset_check(Mesh& m)
{
  u32 const* hc = m.mb->host + COOP_CTL_SLOT;
  // a set that failed leaves its control words standing: zeroed here for
  // the next set's prologue, which appends to list length 0
  auto reset = [&] {
    CK(cudaMemsetAsync(m.mb->dev + COOP_CTL_SLOT, 0, COOP_CTL_WORDS * sizeof(u32), m.s));
  };
  if (hc[6]) {
    reset();
    throw Failure(E_TIMEOUT, "independent set: a grid barrier wait gave up");
  }
  u32 rounds = hc[5];
  last_pass_stats().indset_rounds = rounds;
  // settled: no entity, or the last round left none undecided (the rounds
  // kernel zeroed the list lengths then)
  bool done = rounds == 0 || hc[2 + rounds % 3] == 0;
  if (!done) {
    reset();
    throw Failure(E_NOCONVERGE, "independent set did not settle in 100 rounds");
  }
}

// ---------------------------------------------------------------------------
// expansion and inheritance

template <class T>
__global__ void k_expand_scaled(T const* __restrict__ in, u32 const* __restrict__ offs,
    u32 k, u32 n, u32 width, T* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 f = offs[i] * k, e = offs[i + 1] * k;
  for (u32 j = f; j < e; ++j)
    for (u32 c = 0; c < width; ++c) out[(size_t)j * width + c] = in[(size_t)i * width + c];
}

void expand_scaled(void const* in, u32 const* offs, u32 k, u32 n, u32 width,
    u32 esz, void* out, cudaStream_t s)
{
  if (!n || !width || !k) return;
  PROBE(P_EXPAND, s, 4.0 * (n + 1) + 2.0 * (double)n * width * esz * k);
  u32 const gb = tuned(TK_GATHER_BLOCK);
  if (esz == 1)
    CK(launch_kernel(k_expand_scaled<unsigned char>, dim3(grid_for(n, gb)), dim3(gb), 0, s,
        (unsigned char const*)in, offs, k, n, width, (unsigned char*)out));
  else if (esz == 4)
    CK(launch_kernel(k_expand_scaled<u32>, dim3(grid_for(n, gb)), dim3(gb), 0, s,
        (u32 const*)in, offs, k, n, width, (u32*)out));
  else
    CK(launch_kernel(k_expand_scaled<unsigned long long>, dim3(grid_for(n, gb)), dim3(gb), 0, s,
        (unsigned long long const*)in, offs, k, n, width, (unsigned long long*)out));
  CK_LAUNCH();
}

// Several row expansions in one launch: blockIdx.y picks the job, the x
// blocks stride over its rows (the same copy as k_expand_scaled).
struct ExpandJobs {
  ExpandJob j[8];
};

template <class T>
__device__ inline void copy_rows(void const* in, void* out, u32 i, u32 f, u32 e, u32 width)
{
  T const* src = static_cast<T const*>(in) + (size_t)i * width;
  for (u32 j = f; j < e; ++j) {
    T* dst = static_cast<T*>(out) + (size_t)j * width;
    for (u32 c = 0; c < width; ++c) dst[c] = src[c];
  }
}

// Jobs over every row with k = 1 -- the survivors' copy, one output row or
// none per row, in order: a stream compaction -- of rows of W 32-bit words
// go by warps: a warp takes EXPAND_CHUNKS runs of 32 consecutive rows,
// loads their offsets (one per lane) and their words coalesced, all before
// any store, and stores each word at its row's place, the row's offsets
// coming by shuffle; the kept rows' words stay consecutive, so the stores
// are coalesced too. (A thread per row read and wrote rows of 2-4 words a
// row apart per lane, with one or two loads in flight: a third of DRAM
// peak.)
constexpr u32 EXPAND_CHUNKS = 2;

template <u32 W>
__device__ inline void expand_same_rows(ExpandJob const& jb, u32 warp, u32 nwarps)
{
  u32 const lane = threadIdx.x & 31;
  u32 const* __restrict__ in = static_cast<u32 const*>(jb.in);
  u32 const* __restrict__ in2 = static_cast<u32 const*>(jb.in2);
  u32* __restrict__ out = static_cast<u32*>(jb.out);
  u32* __restrict__ out2 = static_cast<u32*>(jb.out2);
  bool const two = in2 != nullptr;
  for (u32 base = warp * 32 * EXPAND_CHUNKS; base < jb.n; base += nwarps * 32 * EXPAND_CHUNKS) {
    u32 o0[EXPAND_CHUNKS], o1[EXPAND_CHUNKS], a[EXPAND_CHUNKS][W], b[EXPAND_CHUNKS][W];
#pragma unroll
    for (u32 ch = 0; ch < EXPAND_CHUNKS; ++ch) {
      u32 const cb = base + ch * 32;
      u32 const nrows = cb < jb.n ? min(32u, jb.n - cb) : 0u, nw = nrows * W;
      o0[ch] = o1[ch] = 0;
      if (lane < nrows) {
        o0[ch] = jb.offs[cb + lane];
        o1[ch] = jb.offs[cb + lane + 1];
      }
#pragma unroll
      for (u32 it = 0; it < W; ++it) {
        u32 const q = it * 32 + lane;
        if (q < nw) {
          a[ch][it] = in[(size_t)cb * W + q];
          if (two) b[ch][it] = in2[(size_t)cb * W + q];
        }
      }
    }
#pragma unroll
    for (u32 ch = 0; ch < EXPAND_CHUNKS; ++ch) {
      u32 const cb = base + ch * 32;
      u32 const nw = (cb < jb.n ? min(32u, jb.n - cb) : 0u) * W;
#pragma unroll
      for (u32 it = 0; it < W; ++it) {
        u32 const q = it * 32 + lane;
        u32 const row = q / W, c = q - row * W;
        u32 const f = __shfl_sync(0xffffffffu, o0[ch], row & 31);
        u32 const e = __shfl_sync(0xffffffffu, o1[ch], row & 31);
        if (q < nw)
          for (u32 j = f; j < e; ++j) {  // (a row of the survivors' copy has one)
            out[(size_t)j * W + c] = a[ch][it];
            if (two) out2[(size_t)j * W + c] = b[ch][it];
          }
      }
    }
  }
}

// Other jobs (a list of rows, k > 1, wider rows, 1-byte elements): a
// thread per row. (At least three blocks of 512 per SM: at 56 registers
// only four blocks of 256 fit, too few warps to keep the loads in flight.)
__global__ void __launch_bounds__(512, 3) k_expand_many(const __grid_constant__ ExpandJobs jobs)
{
  pdl_wait();
  ExpandJob const jb = jobs.j[blockIdx.y];
  u32 const t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  u32 const words = jb.esz == 4 ? jb.width : jb.esz == 8 ? 2 * jb.width : 0;
  if (words && words <= 4 && !jb.list && jb.k == 1) {
    u32 const warp = t0 / 32, nwarps = stride / 32;
    if (words == 1)
      expand_same_rows<1>(jb, warp, nwarps);
    else if (words == 2)
      expand_same_rows<2>(jb, warp, nwarps);
    else if (words == 3)
      expand_same_rows<3>(jb, warp, nwarps);
    else
      expand_same_rows<4>(jb, warp, nwarps);
    return;
  }
  for (u32 t = t0; t < jb.n; t += stride) {
    u32 const i = jb.list ? jb.list[t] : t;
    u32 f = jb.offs[i] * jb.k, e = jb.offs[i + 1] * jb.k;
    if (jb.esz == 4) {
      copy_rows<u32>(jb.in, jb.out, i, f, e, jb.width);
      if (jb.in2) copy_rows<u32>(jb.in2, jb.out2, i, f, e, jb.width);
    } else if (jb.esz == 8) {
      copy_rows<unsigned long long>(jb.in, jb.out, i, f, e, jb.width);
      if (jb.in2) copy_rows<unsigned long long>(jb.in2, jb.out2, i, f, e, jb.width);
    } else {
      copy_rows<unsigned char>(jb.in, jb.out, i, f, e, jb.width);
      if (jb.in2) copy_rows<unsigned char>(jb.in2, jb.out2, i, f, e, jb.width);
    }
  }
}

void expand_many(std::vector<ExpandJob> const& jobs, cudaStream_t s)
{
  std::vector<ExpandJob> live;
  for (ExpandJob const& jb : jobs)
    if (jb.n && jb.width && jb.k) live.push_back(jb);
  for (size_t at = 0; at < live.size(); at += 8) {
    ExpandJobs pack;
    u32 cnt = (u32)std::min<size_t>(8, live.size() - at), nmax = 0;
    double bytes = 0;
    for (u32 q = 0; q < cnt; ++q) {
      pack.j[q] = live[at + q];
      nmax = std::max(nmax, pack.j[q].n);
      bytes += 4.0 * (pack.j[q].n + 1) + (pack.j[q].in2 ? 4.0 : 2.0) *
          (double)pack.j[q].n * pack.j[q].width * pack.j[q].esz * pack.j[q].k;
    }
    PROBE(P_EXPAND, s, bytes);
    // a grid-stride loop over at most 16 blocks of 256 threads per SM
    // (measured: a block per 256 rows was twice as slow on the 48^3 adapt)
    u32 const gb = tuned(TK_GATHER_BLOCK);
    dim3 grid(std::min<u32>(grid_for(nmax, gb), 148u * 16u * 256u / gb), cnt);
    CK(launch_kernel(k_expand_many, dim3(grid), dim3(gb), 0, s, pack));
    CK_LAUNCH();
  }
}

// class_dim / class_id of the products: every domain of both labels in one
// launch
void inherit_class(Mesh& m, Mesh& out, u32 prod, Doms const& d,
    std::vector<ExpandJob> const* also, std::vector<ExpandJob>* defer)
{
  if (!m.find_tag(0, "class_dim")) {
    if (also && defer)
      defer->insert(defer->end(), also->begin(), also->end());
    else if (also)
      expand_many(*also, m.s);
    return;
  }
  char const* names[2] = {"class_dim", "class_id"};
  u32 nnames = m.find_tag(0, "class_id") ? 2 : 1;
  std::vector<ExpandJob> jobs;
  if (also) jobs = *also;
  u32* data[2] = {nullptr, nullptr};
  u32 nc[2] = {1, 1};
  Tag* t[2] = {nullptr, nullptr};
  for (u32 q = 0; q < nnames; ++q) {
    t[q] = m.find_tag(prod, names[q]);
    if (!t[q]) throw Failure(E_ARG, std::string("missing tag ") + names[q]);
    nc[q] = t[q]->ncomps;
    data[q] = dalloc<u32>((size_t)d.ngo[4] * nc[q], m.s);
  }
  // both labels of a domain dimension in one job when they have the same
  // width (the domain offsets are read once); a domain with a list of its
  // producing entities walks only those
  bool const paired = nnames == 2 && nc[0] == nc[1];
  for (u32 k = 0; k < 4; ++k) {
    if (!d.ndoms[k] || !d.offs[k] || !d.ngen[k]) continue;
    for (u32 q = 0; q < nnames; ++q) {
      Tag* tk = (k == 0) ? t[q] : m.find_tag(k, names[q]);
      if (!tk) continue;
      ExpandJob jb;
      jb.in = tk->data;
      jb.offs = d.offs[k];
      jb.out = data[q] + (size_t)d.ngo[k] * nc[q];
      jb.k = d.scale[k];
      jb.n = d.ndoms[k];
      if (d.list[k]) {
        jb.list = d.list[k];
        jb.n = d.nlist[k];
      }
      jb.width = nc[q];
      jb.esz = 4;
      if (paired && q == 0) {
        Tag* tk2 = (k == 0) ? t[1] : m.find_tag(k, names[1]);
        if (tk2) {
          jb.in2 = tk2->data;
          jb.out2 = data[1] + (size_t)d.ngo[k] * nc[1];
          jobs.push_back(jb);
          break;  // the second label goes with the first
        }
      }
      jobs.push_back(jb);
    }
  }
  if (defer)
    defer->insert(defer->end(), jobs.begin(), jobs.end());
  else
    expand_many(jobs, m.s);
  for (u32 q = 0; q < nnames; ++q) out.add_tag(prod, T_U32, names[q], nc[q], X_NOT, data[q]);
}

void inherit_globals(Mesh& out, u32 d)
{
  out.set_iota_globals(d);
}

__global__ void k_interp_coords(u32 ne, u32 vpe, u32 const* __restrict__ voe,
    double const* __restrict__ x, double* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  // average_element_field (element_field.hpp:9-25)
  double o0 = 0, o1 = 0, o2 = 0;
  for (u32 j = 0; j < vpe; ++j) {
    u32 v = voe[(size_t)i * vpe + j];
    o0 += x[v * 3 + 0];
    o1 += x[v * 3 + 1];
    o2 += x[v * 3 + 2];
  }
  out[i * 3 + 0] = o0 / vpe;
  out[i * 3 + 1] = o1 / vpe;
  out[i * 3 + 2] = o2 / vpe;
}

void interp_coords_to_elems(Mesh& m)
{
  u32 ne = m.count(m.dim), vpe = deg(m.dim, 0);
  double* out = dalloc<double>((size_t)ne * 3, m.s);
  if (ne) {
    CK(launch_kernel(k_interp_coords, dim3(grid_for(ne)), dim3(BLOCK), 0, m.s, ne, vpe, m.ask_down(m.dim, 0),
        m.coords(), out));
    CK_LAUNCH();
  }
  m.add_tag(m.dim, T_F64, "coordinates", 3, X_NOT, out);
}

// ---------------------------------------------------------------------------
// marking (mark.cpp)

__global__ void k_mark_down(u32 n, u32 const* __restrict__ offs, u32 const* __restrict__ adj,
    u32 const* __restrict__ marked, u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 r = 0;
  for (u32 j = offs[i]; j < offs[i + 1]; ++j)
    if (marked[adj[j]]) {
      r = 1;
      break;
    }
  out[i] = r;
}

u32* mark_down(Mesh& m, u32 high, u32 low, u32 const* marked)
{
  u32 n = m.count(low);
  UpAdj const& u = m.ask_up(low, high, false);
  u32* out = dalloc<u32>(n, m.s);
  if (n) {
    CK(launch_kernel(k_mark_down, dim3(grid_for(n)), dim3(BLOCK), 0, m.s, n, u.offs, u.adj, marked, out));
    CK_LAUNCH();
  }
  return out;
}

__global__ void k_mark_up(u32 n, u32 lph, u32 const* __restrict__ loh,
    u32 const* __restrict__ marked, u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 r = 0;
  for (u32 j = 0; j < lph; ++j)
    if (marked[loh[(size_t)i * lph + j]]) {
      r = 1;
      break;
    }
  out[i] = r;
}

u32* mark_up(Mesh& m, u32 low, u32 high, u32 const* marked)
{
  u32 n = m.count(high);
  u32* out = dalloc<u32>(n, m.s);
  if (n) {
    CK(launch_kernel(k_mark_up, dim3(grid_for(n)), dim3(BLOCK), 0, m.s, n, deg(high, low), m.ask_down(high, low),
        marked, out));
    CK_LAUNCH();
  }
  return out;
}

__global__ void k_mark_slivers(u32 n, double const* __restrict__ q, double gq,
    u32 const* __restrict__ voe, u32 vpe, SegView sv, u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (q[i] < gq && (!sv.active || seg_acts(sv, voe[(size_t)i * vpe]))) ? 1u : 0u;
}

// warp-aggregated per-segment count of flagged entities
__global__ void k_seg_tally(u32 n, u32 const* __restrict__ flags, u32 const* __restrict__ voe,
    u32 vpe, u32 const* __restrict__ seg, u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  bool on = i < n && flags[i] != 0;
  u32 mask = __ballot_sync(0xffffffffu, on);
  if (!on) return;
  u32 sg = seg[voe ? voe[(size_t)i * vpe] : i];
  u32 peers = __match_any_sync(mask, sg);
  if ((threadIdx.x & 31) == (u32)(__ffs(peers) - 1)) atomicAdd(&out[sg], (u32)__popc(peers));
}

void seg_tally(Mesh& m, u32 ent_dim, u32 const* flags)
{
  if (!m.seg || !m.ctl || !m.ctl->selected) return;
  u32 n = m.count(ent_dim);
  if (!n) return;
  u32 const* voe = ent_dim ? m.ask_down(ent_dim, 0) : nullptr;
  CK(launch_kernel(k_seg_tally, dim3(grid_for(n)), dim3(BLOCK), 0, m.s, n, flags, voe, deg(ent_dim, 0), m.seg,
      m.ctl->selected));
  CK_LAUNCH();
}

__global__ void k_dual_layer(u32 n, u32 degr, u32 const* __restrict__ dual,
    u32 const* __restrict__ in, u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 r = in[i];
  for (u32 j = 0; j < degr; ++j) {
    u32 e = dual[(size_t)i * degr + j];
    if (e != INV && in[e]) r = 1;
  }
  out[i] = r;
}

// mesh_mark_slivers + mesh_mark_dual_layers (mark.cpp:101-147,218-243)
u32* mark_slivers(Mesh& m, double gq, u32 nlayers)
{
  u32 n = m.count(m.dim);
  double const* q = m.qualities();
  u32* a = dalloc<u32>(n, m.s);
  if (n) {
    SegView sv = m.segview();
    CK(launch_kernel(k_mark_slivers, dim3(grid_for(n)), dim3(BLOCK), 0, m.s, n, q, gq,
        sv.active ? m.ask_down(m.dim, 0) : nullptr, deg(m.dim, 0), sv, a));
    CK_LAUNCH();
  }
  if (!nlayers) return a;
  u32 const* du = m.ask_dual();
  u32* b = dalloc<u32>(n, m.s);
  u32 degr = deg(m.dim, m.dim - 1);
  for (u32 l = 0; l < nlayers; ++l) {
    if (n) {
      CK(launch_kernel(k_dual_layer, dim3(grid_for(n)), dim3(BLOCK), 0, m.s, n, degr, du, a, b));
      CK_LAUNCH();
    }
    std::swap(a, b);
  }
  dev_free(b, m.s);
  return a;
}

}  // namespace osh
