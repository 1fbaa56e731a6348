// Device runtime for the adaptation pass: error state, stream-ordered
// allocation, the decoupled look-back exclusive scan and small array kernels.
#include <algorithm>
#include <cstdlib>
#include <dlfcn.h>
#include <string>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "runtime.hpp"

namespace osh {

namespace {

struct TuneSpec {
  char const* name;
  u32 def;
  u32 allowed[5];
};
TuneSpec const g_tune_spec[TK_NKEYS] = {
    {"carry_group", 8, {4, 8, 16, 0, 0}},
    {"vert_group", 8, {4, 8, 16, 0, 0}},
    {"indset_vert_group", 8, {4, 8, 16, 0, 0}},
    {"indset_edge_group", 4, {1, 2, 4, 8, 0}},
    {"quality_block", 256, {64, 128, 256, 512, 0}},
    {"gather_block", 256, {128, 256, 512, 0, 0}},
    {"scan_items", 16, {8, 16, 0, 0, 0}},
    {"scan_threads", 512, {256, 512, 0, 0, 0}},
    {"indset_blocks", 0, {0, 1, 2, 4, 0}},
    {"small_mesh_elems", 50000, {0, 25000, 50000, 100000, 200000}},
};
std::atomic<u32> g_tune[TK_NKEYS];
std::once_flag g_tune_once;

bool tune_allowed(u32 k, u32 v)
{
  // the list ends at the first 0 after its first entry (0 may be a value)
  TuneSpec const& t = g_tune_spec[k];
  for (u32 i = 0; i < 5; ++i) {
    if (i > 0 && t.allowed[i] == 0) break;
    if (t.allowed[i] == v) return true;
  }
  return false;
}

int tune_find(char const* name)
{
  if (!name) return -1;
  for (u32 k = 0; k < TK_NKEYS; ++k)
    if (std::strcmp(name, g_tune_spec[k].name) == 0) return (int)k;
  return -1;
}

int tune_read_file(char const* path, bool apply)
{
  FILE* f = std::fopen(path, "r");
  if (!f) return E_IO;
  std::vector<std::pair<u32, u32>> sets;
  char line[256];
  int rc = E_OK;
  while (std::fgets(line, sizeof line, f)) {
    char* h = std::strchr(line, '#');
    if (h) *h = 0;
    char name[64];
    unsigned v = 0;
    char extra[8];
    int got = std::sscanf(line, "%63s %u %7s", name, &v, extra);
    if (got <= 0) continue;  // blank or comment
    int k = got == 2 ? tune_find(name) : -1;
    if (k < 0 || !tune_allowed((u32)k, v)) {
      rc = E_ARG;
      break;
    }
    sets.emplace_back((u32)k, (u32)v);
  }
  std::fclose(f);
  if (rc == E_OK && apply)
    for (auto const& kv : sets) g_tune[kv.first].store(kv.second);
  return rc;
}

void tune_init()
{
  std::call_once(g_tune_once, [] {
    for (u32 k = 0; k < TK_NKEYS; ++k) g_tune[k].store(g_tune_spec[k].def);
    char const* env = std::getenv("OSH_B200_TUNING");
    if (env && *env) {
      tune_read_file(env, true);
      return;
    }
    Dl_info info;
    if (dladdr(reinterpret_cast<void*>(&tune_init), &info) && info.dli_fname) {
      std::string p(info.dli_fname);
      size_t slash = p.rfind('/');
      p = (slash == std::string::npos ? std::string(".") : p.substr(0, slash)) + "/tuning.txt";
      tune_read_file(p.c_str(), true);
    }
  });
}

}  // namespace

u32 tuned(TuneKey k)
{
  tune_init();
  return g_tune[k].load(std::memory_order_relaxed);
}

char const* tune_name(u32 k) { return k < TK_NKEYS ? g_tune_spec[k].name : nullptr; }

int tune_set(char const* name, u32 value)
{
  tune_init();
  int k = tune_find(name);
  if (k < 0 || !tune_allowed((u32)k, value)) return E_ARG;
  g_tune[k].store(value);
  return E_OK;
}

int tune_get(char const* name, u32* value)
{
  tune_init();
  int k = tune_find(name);
  if (k < 0) return E_ARG;
  if (value) *value = g_tune[k].load();
  return E_OK;
}

int tune_load(char const* path)
{
  tune_init();
  if (!path) return E_ARG;
  return tune_read_file(path, true);
}

bool pdl_enabled()
{
  static bool const on = [] {
    char const* e = std::getenv("OSH_B200_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}


// ---------------------------------------------------------------------------
// errors

namespace {
thread_local int t_err = 0;
thread_local std::string t_msg;
}  // namespace

void set_error(int code, char const* msg)
{
  t_err = code;
  t_msg = msg ? msg : "";
}
int last_error() { return t_err; }
char const* last_error_message() { return t_msg.c_str(); }
void clear_error()
{
  t_err = 0;
  t_msg.clear();
}

void check_cuda(cudaError_t e, char const* what, char const* file, int line)
{
  if (e == cudaSuccess) return;
  char buf[512];
  snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e),
      file, line);
  throw Failure(e == cudaErrorMemoryAllocation ? E_NOMEM : E_CUDA, buf);
}

// ---------------------------------------------------------------------------
// launch counter (every kernel launch goes through CK_LAUNCH)

namespace {
std::atomic<unsigned long long> g_launches{0};
}
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(); }

namespace {
std::atomic<unsigned long long> g_syncs{0};
std::atomic<unsigned long long> g_sync_ns{0};
std::atomic<unsigned long long> g_allocs{0};
}
unsigned long long sync_count() { return g_syncs.load(); }
void stream_sync(cudaStream_t s)
{
  g_syncs.fetch_add(1, std::memory_order_relaxed);
  auto t0 = std::chrono::steady_clock::now();
  CK(cudaStreamSynchronize(s));
  auto dt = std::chrono::steady_clock::now() - t0;
  g_sync_ns.fetch_add((unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
      dt).count(), std::memory_order_relaxed);
}
void host_stats(unsigned long long* allocs, double* sync_seconds)
{
  if (allocs) *allocs = g_allocs.load();
  if (sync_seconds) *sync_seconds = g_sync_ns.load() * 1e-9;
}

// ---------------------------------------------------------------------------
// probes

namespace {
struct ProbeState {
  u32 mask = 0;
  struct Rec {
    cudaEvent_t a, b;
    double bytes;
  };
  std::vector<Rec> recs[P_NPROBES];
  u32 launches[P_NPROBES] = {};
  double ms[P_NPROBES] = {};
  double bytes[P_NPROBES] = {};
  std::mutex mu;
};
ProbeState& probes()
{
  static ProbeState p;
  return p;
}
char const* const g_probe_names[P_NPROBES] = {"reflect_down", "up_count", "up_fill",
    "up_rank", "exscan", "elem_quality", "refine_candidates", "refine_quality",
    "indset_round", "coarsen_quality", "swap_quality", "refine_topology",
    "collapse_to_ent", "expand", "carry_down", "carry_up", "carry_up_fill"};
}  // namespace

char const* probe_name(u32 id) { return id < P_NPROBES ? g_probe_names[id] : nullptr; }

namespace {
std::once_flag g_fp32_once[64];
Fp32Stats* g_fp32[64] = {};
}

Fp32Stats* fp32_stats_dev()
{
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw Failure(E_ARG, "device index out of range");
  std::call_once(g_fp32_once[dev], [dev]() {
    void* p = nullptr;
    CK(cudaMalloc(&p, sizeof(Fp32Stats)));
    CK(cudaMemset(p, 0, sizeof(Fp32Stats)));
    g_fp32[dev] = static_cast<Fp32Stats*>(p);
  });
  return g_fp32[dev];
}

void fp32_stats_read(unsigned long long* decided, unsigned long long* rechecked,
    double* max_err, unsigned* bound_exceeded)
{
  Fp32Stats h;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(&h, fp32_stats_dev(), sizeof(h), cudaMemcpyDeviceToHost));
  float e;
  std::memcpy(&e, &h.max_err_bits, sizeof(e));
  if (decided) *decided = h.decided;
  if (rechecked) *rechecked = h.rechecked;
  if (max_err) *max_err = e;
  if (bound_exceeded) *bound_exceeded = h.bound_exceeded;
}

void fp32_audit_read(unsigned long long* audited, unsigned long long* flips,
    unsigned long long* checked)
{
  Fp32Stats h;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(&h, fp32_stats_dev(), sizeof(h), cudaMemcpyDeviceToHost));
  if (audited) *audited = h.audited;
  if (flips) *flips = h.flips;
  if (checked) *checked = h.checked;
}

// the counters return to zero; the audit switch is kept
void fp32_stats_reset()
{
  CK(cudaDeviceSynchronize());
  Fp32Stats* d = fp32_stats_dev();
  unsigned audit = 0;
  CK(cudaMemcpy(&audit, &d->audit, sizeof(audit), cudaMemcpyDeviceToHost));
  Fp32Stats z;
  std::memset(&z, 0, sizeof(z));
  z.audit = audit;
  CK(cudaMemcpy(d, &z, sizeof(z), cudaMemcpyHostToDevice));
}

void fp32_set_audit(bool on)
{
  CK(cudaDeviceSynchronize());
  unsigned v = on ? 1u : 0u;
  CK(cudaMemcpy(&fp32_stats_dev()->audit, &v, sizeof(v), cudaMemcpyHostToDevice));
}

void probe_enable(u32 mask) { probes().mask = mask; }

static void probe_resolve(ProbeState& p)
{
  for (u32 i = 0; i < P_NPROBES; ++i) {
    for (auto& r : p.recs[i]) {
      float t = 0;
      CK(cudaEventSynchronize(r.b));
      CK(cudaEventElapsedTime(&t, r.a, r.b));
      p.launches[i] += 1;
      p.ms[i] += t;
      p.bytes[i] += r.bytes;
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
    p.recs[i].clear();
  }
}

void probe_reset()
{
  ProbeState& p = probes();
  std::lock_guard<std::mutex> g(p.mu);
  probe_resolve(p);
  for (u32 i = 0; i < P_NPROBES; ++i) {
    p.launches[i] = 0;
    p.ms[i] = 0;
    p.bytes[i] = 0;
  }
}

void probe_read(u32 id, u32* launches, double* ms, double* bytes)
{
  ProbeState& p = probes();
  std::lock_guard<std::mutex> g(p.mu);
  probe_resolve(p);
  *launches = p.launches[id];
  *ms = p.ms[id];
  *bytes = p.bytes[id];
}

ProbeScope::ProbeScope(u32 i, cudaStream_t st, double by) : id(i), bytes(by), s(st)
{
  if (!((probes().mask >> id) & 1u)) return;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  CK(cudaEventRecord(a, s));
}

ProbeScope::~ProbeScope()
{
  if (!a) return;
  cudaEventRecord(b, s);
  ProbeState& p = probes();
  std::lock_guard<std::mutex> g(p.mu);
  p.recs[id].push_back({a, b, bytes});
}

// ---------------------------------------------------------------------------
// allocation: the device's default memory pool, never trimmed between passes

namespace {
std::once_flag g_pool_once[64];
}

static void setup_pool()
{
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::call_once(g_pool_once[dev & 63], [dev]() {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      unsigned long long thr = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
  });
}

void* dev_alloc(size_t bytes, cudaStream_t s)
{
  setup_pool();
  void* p = nullptr;
  if (bytes < 16) bytes = 16;
  g_allocs.fetch_add(1, std::memory_order_relaxed);
  cudaError_t e = cudaMallocAsync(&p, bytes, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    char buf[128];
    snprintf(buf, sizeof(buf), "device allocation of %zu bytes failed", bytes);
    throw Failure(E_NOMEM, buf);
  }
  return p;
}

void pool_reserve(unsigned long long bytes)
{
  setup_pool();
  if (!bytes) return;
  void* p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, bytes, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Failure(E_NOMEM, "could not reserve the requested device memory");
  }
  CK(cudaFreeAsync(p, 0));
  CK(cudaStreamSynchronize(0));
}

void pool_stats(unsigned long long* reserved, unsigned long long* used,
    unsigned long long* used_high, int reset_high)
{
  setup_pool();
  int dev = 0;
  CK(cudaGetDevice(&dev));
  cudaMemPool_t pool;
  CK(cudaDeviceGetDefaultMemPool(&pool, dev));
  unsigned long long r = 0, u = 0, h = 0;
  CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r));
  CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u));
  CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &h));
  if (reserved) *reserved = r;
  if (used) *used = u;
  if (used_high) *used_high = h;
  if (reset_high) {
    unsigned long long zero = 0;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero));
  }
}

void dev_free(void* p, cudaStream_t s)
{
  if (p) CK(cudaFreeAsync(p, s));
}

namespace {
// a pinned word per host thread for read_u32: a copy into pageable memory
// goes through the driver's staging buffer and takes several times longer.
// Words go back to a process-wide free list when their thread ends (pinning
// and unpinning memory each take a driver call that can wait for the
// device, which short-lived worker threads would pay every time).
std::mutex g_words_mu;
std::vector<u32*>& free_words()
{
  static std::vector<u32*>* v = new std::vector<u32*>();  // lives to exit
  return *v;
}
struct PinnedWord {
  u32* p = nullptr;
  ~PinnedWord()
  {
    if (!p) return;
    std::lock_guard<std::mutex> g(g_words_mu);
    free_words().push_back(p);
  }
  u32* get()
  {
    if (p) return p;
    {
      std::lock_guard<std::mutex> g(g_words_mu);
      if (!free_words().empty()) {
        p = free_words().back();
        free_words().pop_back();
        return p;
      }
    }
    CK(cudaMallocHost(&p, 64));
    return p;
  }
};
thread_local PinnedWord t_word;
}  // namespace

void* pinned_scratch() { return t_word.get(); }

u32 read_u32(u32 const* d, cudaStream_t s)
{
  u32* h = t_word.get();
  CK(cudaMemcpyAsync(h, d, sizeof(u32), cudaMemcpyDeviceToHost, s));
  stream_sync(s);
  return *h;
}

double read_f64(double const* d, cudaStream_t s)
{
  double* h = static_cast<double*>(pinned_scratch());
  CK(cudaMemcpyAsync(h, d, sizeof(double), cudaMemcpyDeviceToHost, s));
  stream_sync(s);
  return *h;
}

void Mailbox::init(cudaStream_t s)
{
  if (host) return;
  // the sequence word on a line of its own
  CK(cudaMallocHost(&host, (SEQ_SLOT + 32) * sizeof(u32)));
  std::memset(host, 0, (SEQ_SLOT + 32) * sizeof(u32));
  void* hd = nullptr;
  CK(cudaHostGetDevicePointer(&hd, host, 0));
  hdev = static_cast<u32*>(hd);
  seq = 0;
  dev = dalloc<u32>(64, s);
  clear(s);
}

void Mailbox::release()
{
  if (host) cudaFreeHost(host);
  if (dev) cudaFree(dev);
  host = nullptr;
  hdev = nullptr;
  dev = nullptr;
}

void Mailbox::clear(cudaStream_t s)
{
  CK(cudaMemsetAsync(dev, 0, 64 * sizeof(u32), s));
}

// dst: the host words' device address; seq_at: the sequence word's
__global__ void k_mailbox_post(u32 const* __restrict__ src, u32 n, u32* dst, u32* seq_at,
    u32 seq)
{
  pdl_wait();
  u32 i = threadIdx.x;
  if (i < n) {
    reinterpret_cast<volatile u32*>(dst)[i] = src[i];
    __threadfence_system();  // this word reaches the host before the sequence word
  }
  __syncthreads();
  if (i == 0) *reinterpret_cast<volatile u32*>(seq_at) = seq;
}

u32 const* Mailbox::read(cudaStream_t s, u32 const* src, u32 nwords)
{
  if (nwords > 16) throw Failure(E_ARG, "mailbox read: at most 16 words");
  post(s, src, nwords, READ_SLOT);
  return host + READ_SLOT;
}

void Mailbox::fetch(cudaStream_t s, u32 nslots)
{
  post(s, dev, nslots > 64 ? 64 : nslots, 0);
}

void Mailbox::post(cudaStream_t s, u32 const* src, u32 nslots, u32 at)
{
  u32 const want = ++seq;
  g_syncs.fetch_add(1, std::memory_order_relaxed);
  auto t0 = std::chrono::steady_clock::now();
  CK(launch_kernel(k_mailbox_post, dim3(1), dim3(64), 0, s, src, nslots, hdev + at,
      hdev + SEQ_SLOT, want));
  CK_LAUNCH();
  volatile u32* flag = host + SEQ_SLOT;
  for (u64 it = 1; *flag != want; ++it) {
    if ((it & 255) != 0) continue;
    // now and then: a failed stream ends the wait with its error; a drained
    // stream whose word has not arrived (it should have) falls back to a
    // copy and a synchronisation
    cudaError_t st = cudaStreamQuery(s);
    if (st == cudaErrorNotReady) continue;
    CK(st);
    if (*flag == want) break;
    CK(cudaMemcpyAsync(host + at, src, nslots * sizeof(u32), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    break;
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  auto dt = std::chrono::steady_clock::now() - t0;
  g_sync_ns.fetch_add((unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
      dt).count(), std::memory_order_relaxed);
}

// ---------------------------------------------------------------------------
// exclusive scan, single pass with decoupled look-back.
//
// Tiles are claimed through an atomic ticket, so every tile a block waits on
// was claimed (and is running or done) before it. Each tile publishes its
// aggregate, then walks back over predecessors until it meets an inclusive
// prefix. The walk is bounded: after spin_limit empty polls (SCAN_SPIN_LIMIT
// in every scan the passes issue) it sets the scratch's error word, which
// the host reads for that stream (check_device_timeouts), and stops instead
// of spinning forever.

// Tiles of SCAN_T threads (the tuning table's scan_threads, 256 or 512)
// times SCAN_ITEMS items (scan_items, 8 or 16). With 8192-element tiles a
// 2M-element scan has 256 tiles, so a tile's look-back meets a published
// prefix within a few steps (with 2048-element tiles the chain of
// look-backs, not bandwidth, set the time of the adapt's scans). Scratch
// is sized for the smallest tile, so every shape fits.
constexpr int SCAN_MIN_TILE = 256 * 8;
constexpr unsigned long long FLAG_AGG = 1ull << 62;
constexpr unsigned long long FLAG_PRE = 2ull << 62;
constexpr u32 SCAN_SPIN_LIMIT = 1u << 24;

// Several independent scans in one launch. Job j scans its `in` (mode 0),
// the survivors of an offsets array, (in[i + 1] == in[i]) (mode 1,
// uints_negate_offsets, ints.cpp:227-235), or the entries stamped with its
// stamp, (in[i] == stamp) (mode 2), into out[0..n] with the total at
// out[n] (and in *total_to when given); newid (optional, for 0/1 items)
// receives out[i] where item i is 1 and INV where it is 0 -- each old
// entity's new id when the items mark survivors. Tiles are numbered across
// the jobs (job j owns tiles tile0[j] .. tile0[j + 1] - 1, one at least) and
// claimed through one ticket, so a look-back, which stops at its job's
// first tile, only waits on tiles claimed before it. Independent scans of a
// pass share a launch, and their look-back chains overlap.
template <int SCAN_T, int SCAN_ITEMS>
__global__ void __launch_bounds__(SCAN_T)
k_exscan(ScanJobs jobs, unsigned long long* status, u32* ticket_and_err, u32 spin_limit)
{
  pdl_wait();
  constexpr int SCAN_THREADS = SCAN_T, SCAN_WARPS = SCAN_T / 32;
  __shared__ u32 s_tile;
  __shared__ u32 s_warp[SCAN_WARPS];
  __shared__ u32 s_prefix;
  constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
  __shared__ u32 s_buf[SCAN_TILE + SCAN_TILE / 32];
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket_and_err, 1u);
  __syncthreads();
  u32 const tile = s_tile;
  u32 const ntiles = jobs.tile0[jobs.njobs];
  if (tile >= ntiles) return;
  u32 jn = 0;
  while (jn + 1 < jobs.njobs && tile >= jobs.tile0[jn + 1]) ++jn;
  ScanJob const job = jobs.j[jn];
  u32 const first = jobs.tile0[jn], last = jobs.tile0[jn + 1] - 1;
  u32 const* __restrict__ in = job.in;
  u32 const n = job.n;
  bool const mode1 = job.mode == 1, mode2 = job.mode == 2;
  u32 const stamp = job.stamp;
  size_t const base = (size_t)(tile - first) * SCAN_TILE;
  // coalesced load into shared memory (padded to avoid bank conflicts)
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    u32 li = k * SCAN_THREADS + threadIdx.x;
    size_t gi = base + li;
    u32 v = 0;
    if (gi < n)
      v = mode2 ? (in[gi] == stamp ? 1u : 0u)
                : !mode1 ? in[gi] : (in[gi + 1] == in[gi] ? 1u : 0u);
    s_buf[li + (li >> 5)] = v;
  }
  __syncthreads();
  u32 v[SCAN_ITEMS];
  u32 sum = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    u32 li = threadIdx.x * SCAN_ITEMS + k;
    v[k] = s_buf[li + (li >> 5)];
    sum += v[k];
  }
  u32 const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u32 x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    u32 y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (u32)o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    u32 w = lane < SCAN_WARPS ? s_warp[lane] : 0u;
#pragma unroll
    for (int o = 1; o < SCAN_WARPS; o <<= 1) {
      u32 y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= (u32)o) w += y;
    }
    if (lane < SCAN_WARPS) s_warp[lane] = w;
  }
  __syncthreads();
  u32 const thread_excl = (warp ? s_warp[warp - 1] : 0u) + x - sum;
  u32 const total = s_warp[SCAN_WARPS - 1];
  if (warp == 0) {
    // warp-cooperative look-back: lane l inspects tile (p - l)
    u32 prefix = 0;
    if (tile == first) {
      if (lane == 0) atomicExch(&status[tile], FLAG_PRE | (unsigned long long)total);
    } else {
      if (lane == 0) atomicExch(&status[tile], FLAG_AGG | (unsigned long long)total);
      int p = (int)tile - 1;
      u32 spins = 0;
      bool gave_up = false;
      for (;;) {
        int idx = p - (int)lane;
        unsigned long long st = FLAG_PRE;  // before the job's first tile: empty
        if (idx >= (int)first) st = *((volatile unsigned long long*)&status[idx]);
        while (__any_sync(0xffffffffu, (st >> 62) == 0)) {
          if (++spins > spin_limit) {
            gave_up = true;
            break;
          }
          if (idx >= (int)first && (st >> 62) == 0)
            st = *((volatile unsigned long long*)&status[idx]);
        }
        if (gave_up) {
          if (lane == 0) atomicOr(&ticket_and_err[1], 1u);
          break;
        }
        u32 pre = __ballot_sync(0xffffffffu, (st & (3ull << 62)) == FLAG_PRE);
        u32 stop = pre ? (u32)(__ffs(pre) - 1) : 31u;
        u32 val = (lane <= stop) ? (u32)st : 0u;
#pragma unroll
        for (int o = 16; o; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
        prefix += val;
        if (pre) break;
        p -= 32;
      }
      if (lane == 0) atomicExch(&status[tile], FLAG_PRE | (unsigned long long)(prefix + total));
    }
    if (lane == 0) s_prefix = prefix;
  }
  __syncthreads();
  u32* __restrict__ out = job.out;
  u32* __restrict__ newid = job.newid;
  u32* __restrict__ list = job.list;
  u32* __restrict__ comp = job.comp;
  u32* __restrict__ comp_newid = job.comp_newid;
  // jobs that need each item's mark keep it in bit 31 of its staged prefix
  // (their prefixes count marked entities: below 2^31), so the store phase
  // does not read the items again
  bool const need_on = newid || list || comp_newid;
  constexpr u32 ON_BIT = 0x80000000u;
  u32 run = s_prefix + thread_excl;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    u32 li = threadIdx.x * SCAN_ITEMS + k;
    s_buf[li + (li >> 5)] = run | (need_on && v[k] ? ON_BIT : 0u);
    run += v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    u32 li = k * SCAN_THREADS + threadIdx.x;
    size_t gi = base + li;
    if (gi < n) {
      u32 const w = s_buf[li + (li >> 5)];
      u32 const o = need_on ? w & ~ON_BIT : w;
      out[gi] = o;
      if (comp) comp[gi] = (u32)gi - o;
      if (need_on) {
        bool const on = (w & ON_BIT) != 0;
        if (newid) newid[gi] = on ? o : INV;
        if (list && on) list[o] = (u32)gi;
        if (comp_newid) comp_newid[gi] = on ? INV : (u32)gi - o;
      }
    }
  }
  if (tile == last && threadIdx.x == 0) {
    out[n] = s_prefix + total;
    if (comp) comp[n] = n - (s_prefix + total);
    if (job.total_to) *job.total_to = s_prefix + total;
  }
  // The last tile to finish returns the scratch to zero for the next scan
  // on the stream: every other tile has counted itself done, so no look-back
  // reads a status word any more.
  __shared__ u32 s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&ticket_and_err[2], 1u) == ntiles - 1 ? 1u : 0u;
  }
  __syncthreads();
  if (s_last) {
    for (u32 t = threadIdx.x; t < ntiles; t += blockDim.x) status[t] = 0ull;
    __syncthreads();
    if (threadIdx.x == 0) {
      ticket_and_err[0] = 0;
      ticket_and_err[2] = 0;
      __threadfence();
    }
  }
}

namespace {
// Scratch of the scans issued on each stream ([ticket, error, done, pad]
// then two words per tile), zero between scans: the scan kernel's last tile
// clears it, so no scan pays for a memset. Scans on one stream run one
// after another; each stream has its own, freed by release_stream_scratch
// when the stream goes.
struct ScanScratch {
  u32* p = nullptr;
  size_t words = 0;
};
std::mutex g_scan_mu;
std::map<std::pair<int, cudaStream_t>, ScanScratch>& scan_scratches()
{
  static auto* m = new std::map<std::pair<int, cudaStream_t>, ScanScratch>();
  return *m;
}

u32* stream_scan_scratch(size_t words, cudaStream_t s)
{
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(g_scan_mu);
  auto& all = scan_scratches();
  ScanScratch& sc = all[{dev, s}];
  if (sc.words < words) {
    size_t want = std::max(words, (size_t)4096);
    if (sc.p) CK(cudaFreeAsync(sc.p, s));
    sc.p = nullptr;
    sc.words = 0;
    void* q = nullptr;
    CK(cudaMallocAsync(&q, want * sizeof(u32), s));
    CK(cudaMemsetAsync(q, 0, want * sizeof(u32), s));
    sc.p = static_cast<u32*>(q);
    sc.words = want;
  }
  return sc.p;
}
}  // namespace

namespace {
// Per-stream scratch kept between calls, one per key (what it holds); see
// stream_zero_scratch and stream_marks
struct KeptScratch {
  u32* p = nullptr;
  size_t words = 0;
  u32 gen = 0;
};
std::mutex g_kept_mu;
using KeptKey = std::tuple<int, cudaStream_t, u32>;
std::map<KeptKey, KeptScratch>& kept_scratches()
{
  static auto* m = new std::map<KeptKey, KeptScratch>();
  return *m;
}

// at least `words` words for (this device, s, key), zeroed when (re)made
KeptScratch& kept_scratch(u32 key, size_t words, cudaStream_t s)
{
  int dev = 0;
  CK(cudaGetDevice(&dev));
  auto& all = kept_scratches();
  KeptScratch& sc = all[{dev, s, key}];
  if (sc.words < words) {
    size_t want = std::max(words + words / 4, (size_t)4096);
    if (sc.p) CK(cudaFreeAsync(sc.p, s));
    void* q = nullptr;
    CK(cudaMallocAsync(&q, want * sizeof(u32), s));
    CK(cudaMemsetAsync(q, 0, want * sizeof(u32), s));
    sc.p = static_cast<u32*>(q);
    sc.words = want;
    sc.gen = 0;
  }
  return sc;
}
}  // namespace

u32 resident_blocks_of(void const* kernel, u32 block, size_t smem)
{
  static std::mutex mu;
  static auto* cache = new std::map<std::tuple<void const*, u32, size_t, int>, u32>();
  int dev = 0;
  CK(cudaGetDevice(&dev));
  auto const key = std::make_tuple(kernel, block, smem, dev);
  std::lock_guard<std::mutex> g(mu);
  auto it = cache->find(key);
  if (it != cache->end()) return it->second;
  int per_sm = 0, sms = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, (int)block, smem));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  u32 const n = (u32)std::max(1, per_sm) * (u32)std::max(1, sms);
  (*cache)[key] = n;
  return n;
}

void release_stream_scratch(cudaStream_t s)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  {
    std::lock_guard<std::mutex> g(g_scan_mu);
    auto& all = scan_scratches();
    auto it = all.find({dev, s});
    if (it != all.end()) {
      if (it->second.p) cudaFreeAsync(it->second.p, s);
      all.erase(it);
    }
  }
  std::lock_guard<std::mutex> g(g_kept_mu);
  auto& all = kept_scratches();
  for (auto it = all.lower_bound(KeptKey{dev, s, 0}); it != all.end() &&
       std::get<0>(it->first) == dev && std::get<1>(it->first) == s;) {
    if (it->second.p) cudaFreeAsync(it->second.p, s);
    it = all.erase(it);
  }
}

u32* stream_zero_scratch(u32 key, size_t words, cudaStream_t s)
{
  std::lock_guard<std::mutex> g(g_kept_mu);
  return kept_scratch(key, words, s).p;
}

u32* stream_marks(u32 key, size_t words, cudaStream_t s, u32* gen)
{
  std::lock_guard<std::mutex> g(g_kept_mu);
  KeptScratch& sc = kept_scratch(key, words, s);
  if (++sc.gen == 0) {  // wrapped: no stamp of old may pass for the new one
    CK(cudaMemsetAsync(sc.p, 0, sc.words * sizeof(u32), s));
    sc.gen = 1;
  }
  *gen = sc.gen;
  return sc.p;
}

namespace {
// tiles of a job (one at least: an empty scan still writes out[0] = 0)
u32 job_tiles(u32 n, u32 tile) { return n ? ceil_div(n, (u64)tile) : 1u; }

// a tile's shape: threads (256 or 512) x items per thread (8 or 16)
struct ScanShape {
  u32 threads, items;
  u32 tile() const { return threads * items; }
};
ScanShape tuned_scan_shape() { return {tuned(TK_SCAN_THREADS), tuned(TK_SCAN_ITEMS)}; }

void launch_scan_jobs(ScanJobs const& jobs, ScanShape sh, u32* scratch, u32 spin_limit,
    cudaStream_t s)
{
  u32 const ntiles = jobs.tile0[jobs.njobs];
  auto k = sh.threads == 256 ? (sh.items == 8 ? k_exscan<256, 8> : k_exscan<256, 16>)
                             : (sh.items == 8 ? k_exscan<512, 8> : k_exscan<512, 16>);
  CK(launch_kernel(k, dim3(ntiles), dim3(sh.threads), 0, s, jobs,
      reinterpret_cast<unsigned long long*>(scratch + 4), scratch, spin_limit));
  CK_LAUNCH();
}
}  // namespace

void exscan_jobs(ScanJob const* jobs, u32 njobs, cudaStream_t s)
{
  ScanShape const sh = tuned_scan_shape();
  u32 const tile = sh.tile();
  for (u32 at = 0; at < njobs; at += MAX_SCAN_JOBS) {
    ScanJobs pack;
    pack.njobs = std::min<u32>(MAX_SCAN_JOBS, njobs - at);
    pack.tile0[0] = 0;
    double bytes = 0;
    for (u32 q = 0; q < pack.njobs; ++q) {
      pack.j[q] = jobs[at + q];
      pack.tile0[q + 1] = pack.tile0[q] + job_tiles(pack.j[q].n, tile);
      bytes += 8.0 * pack.j[q].n + 4.0 + (pack.j[q].newid ? 4.0 * pack.j[q].n : 0.0) +
          (pack.j[q].comp ? 4.0 * pack.j[q].n : 0.0) + (pack.j[q].comp_newid ? 4.0 * pack.j[q].n : 0.0);
    }
    // [ticket, error, done, pad][status per tile], zero on entry
    u32* scratch = stream_scan_scratch(4 + 2 * (size_t)pack.tile0[pack.njobs], s);
    PROBE(P_EXSCAN, s, bytes);
    launch_scan_jobs(pack, sh, scratch, SCAN_SPIN_LIMIT, s);
  }
}

void exscan_u32(u32 const* in, u32* out, u32 n, cudaStream_t s, u32* total_to, u32* newid)
{
  ScanJob j{in, out, total_to, newid, n, 0};
  exscan_jobs(&j, 1, s);
}

// The scans of one stream record a look-back that gave up in word 1 of that
// stream's scratch (the last tile clears words 0 and 2 only), so a stream's
// check sees its own scans' timeouts and no other stream's.
void check_device_timeouts(cudaStream_t s)
{
  int dev = 0;
  CK(cudaGetDevice(&dev));
  u32* p = nullptr;
  {
    std::lock_guard<std::mutex> g(g_scan_mu);
    auto& all = scan_scratches();
    auto it = all.find({dev, s});
    if (it != all.end()) p = it->second.p;
  }
  if (!p) return;
  u32* h = static_cast<u32*>(pinned_scratch());
  CK(cudaMemcpyAsync(h, p + 1, sizeof(u32), cudaMemcpyDeviceToHost, s));
  stream_sync(s);
  if (*h) {
    CK(cudaMemsetAsync(p + 1, 0, sizeof(u32), s));
    stream_sync(s);
    throw Failure(E_TIMEOUT, "a bounded device wait gave up (scan look-back)");
  }
}

int selftest_scan_wait(u32 spin_limit)
{
  // Two tiles, the ticket counter starting at 1: the block that takes tile
  // 1 waits for tile 0, which no block takes, until spin_limit polls have
  // gone by; the block that takes ticket 2 has no tile and returns.
  cudaStream_t s = nullptr;
  CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  u32 const n = 2 * 512 * 16, ntiles = 2;
  size_t words = (size_t)(n + 1) * 2 + 4 + 2 * ntiles + 4;  // + alignment room
  u32* buf = nullptr;
  CK(cudaMalloc(&buf, words * sizeof(u32)));
  u32* in = buf;
  u32* out = buf + n + 1;
  u32* scratch = buf + 2 * (size_t)(n + 1);
  scratch += (4 - (reinterpret_cast<uintptr_t>(scratch) / 4) % 4) % 4;  // 16-byte aligned
  CK(cudaMemsetAsync(buf, 0, words * sizeof(u32), s));
  u32 one = 1;
  CK(cudaMemcpyAsync(scratch, &one, sizeof(u32), cudaMemcpyHostToDevice, s));
  ScanJobs pack;
  pack.njobs = 1;
  pack.tile0[0] = 0;
  pack.tile0[1] = ntiles;
  pack.j[0] = ScanJob{in, out, nullptr, nullptr, n, 0};
  launch_scan_jobs(pack, ScanShape{512, 16}, scratch, spin_limit, s);
  u32 err = 0;
  CK(cudaMemcpyAsync(&err, scratch + 1, sizeof(u32), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaFree(buf));
  CK(cudaStreamDestroy(s));
  return err ? E_TIMEOUT : E_OK;
}

size_t exscan_scratch_words(u32 n)
{
  return 4 + 2 * (size_t)ceil_div(n ? n : 1, SCAN_MIN_TILE);
}

void exscan_u32_scratch(u32 const* in, u32* out, u32 n, u32* scratch, cudaStream_t s)
{
  if (reinterpret_cast<uintptr_t>(scratch) % 16 != 0)
    throw Failure(E_ARG, "scan scratch must start on a 16-byte boundary");
  ScanShape const sh = tuned_scan_shape();
  CK(cudaMemsetAsync(scratch, 0, exscan_scratch_words(n) * sizeof(u32), s));
  ScanJobs pack;
  pack.njobs = 1;
  pack.tile0[0] = 0;
  pack.tile0[1] = job_tiles(n, sh.tile());
  pack.j[0] = ScanJob{in, out, nullptr, nullptr, n, 0};
  launch_scan_jobs(pack, sh, scratch, SCAN_SPIN_LIMIT, s);
}

u32* exscan_new(u32 const* in, u32 n, cudaStream_t s, u32* total_to, u32* newid)
{
  u32* out = dalloc<u32>((size_t)n + 1, s);
  exscan_u32(in, out, n, s, total_to, newid);
  return out;
}

u32* negate_offsets(u32 const* offs, u32 n, cudaStream_t s, u32* total_to, u32* newid)
{
  u32* o = dalloc<u32>((size_t)n + 1, s);
  ScanJob j{offs, o, total_to, newid, n, 1};
  exscan_jobs(&j, 1, s);
  return o;
}

__global__ void k_fill(u32* a, u32 n, u32 v)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

void fill_u32(u32* a, u32 n, u32 v, cudaStream_t s)
{
  if (!n) return;
  CK(launch_kernel(k_fill, dim3(grid_for(n)), dim3(BLOCK), 0, s, a, n, v));
  CK_LAUNCH();
}

__global__ void k_iota(u32* a, u32 n, u32 stride)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i * stride;
}

void iota_u32(u32* a, u32 n, u32 stride, cudaStream_t s)
{
  if (!n) return;
  CK(launch_kernel(k_iota, dim3(grid_for(n)), dim3(BLOCK), 0, s, a, n, stride));
  CK_LAUNCH();
}

__global__ void k_iota64(u64* a, u32 n)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

void iota_u64(u64* a, u32 n, cudaStream_t s)
{
  if (!n) return;
  CK(launch_kernel(k_iota64, dim3(grid_for(n)), dim3(BLOCK), 0, s, a, n));
  CK_LAUNCH();
}

template <class T>
__global__ void k_expand(T const* __restrict__ in, u32 const* __restrict__ offs,
    u32 n, u32 width, T* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 f = offs[i], e = offs[i + 1];
  for (u32 j = f; j < e; ++j)
    for (u32 k = 0; k < width; ++k) out[(size_t)j * width + k] = in[(size_t)i * width + k];
}

void expand_rows(void const* in, u32 const* offs, u32 n, u32 width, u32 esz,
    void* out, cudaStream_t s)
{
  if (!n || !width) return;
  PROBE(P_EXPAND, s, 4.0 * (n + 1) + 2.0 * (double)n * width * esz);
  switch (esz) {
    case 1:
      CK(launch_kernel(k_expand<unsigned char>, dim3(grid_for(n)), dim3(BLOCK), 0, s, 
          (unsigned char const*)in, offs, n, width, (unsigned char*)out));
      break;
    case 4:
      CK(launch_kernel(k_expand<u32>, dim3(grid_for(n)), dim3(BLOCK), 0, s, (u32 const*)in, offs, n, width, (u32*)out));
      break;
    default:
      CK(launch_kernel(k_expand<unsigned long long>, dim3(grid_for(n)), dim3(BLOCK), 0, s, 
          (unsigned long long const*)in, offs, n, width, (unsigned long long*)out));
      break;
  }
  CK_LAUNCH();
}

__global__ void k_max_u32(u32 const* __restrict__ a, u32 n, u32* out)
{
  pdl_wait();
  u32 m = 0;
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    m = max(m, a[i]);
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

u32 max_u32(u32 const* a, u32 n, cudaStream_t s)
{
  if (!n) return 0;
  u32* d = dalloc<u32>(1, s);
  CK(cudaMemsetAsync(d, 0, sizeof(u32), s));
  u32 g = grid_for(n);
  if (g > 4096) g = 4096;
  CK(launch_kernel(k_max_u32, dim3(g), dim3(BLOCK), 0, s, a, n, d));
  CK_LAUNCH();
  u32 v = read_u32(d, s);
  dev_free(d, s);
  return v;
}

}  // namespace osh
