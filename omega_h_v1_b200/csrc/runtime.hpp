// Host-callable device primitives used by every pass: scans, reductions,
// fills, compaction by offsets. All work is issued on the caller's stream.
#pragma once

#include "common.cuh"

namespace osh {

// Launch shapes chosen by the tuner (omega_h_v1_b200/tune.py, which times
// each candidate with CUDA events on a mid-size adapt and writes the table).
// Every key has a default and a set of allowed values; the table is read
// once, from the file named by OSH_B200_TUNING or else tuning.txt beside
// the library ("name value" lines, # comments). Any allowed value gives the
// same meshes: only the launch shapes change.
enum TuneKey : u32 {
  TK_CARRY_GROUP = 0,    // lanes per long carried upward row: 4, 8, 16
  TK_VERT_GROUP,         // lanes per vertex row, coarsening vertex kernels: 4, 8, 16
  TK_INDSET_VERT_GROUP,  // lanes per vertex, independent-set rounds: 4, 8, 16
  TK_INDSET_EDGE_GROUP,  // lanes per edge (3D), independent-set rounds: 1, 2, 4, 8
  TK_QUALITY_BLOCK,      // threads per block, quality kernels: 64, 128, 256, 512
  TK_GATHER_BLOCK,       // threads per block, carry / search / copy kernels: 128, 256, 512
  TK_SCAN_ITEMS,         // items per thread of a scan tile: 8, 16
  TK_SCAN_THREADS,       // threads per scan tile: 256, 512
  TK_INDSET_BLOCKS,      // blocks per SM of the one-launch independent set (each
                         // round ends in a grid barrier that every block joins;
                         // 0: as many as fit): 0, 1, 2, 4
  TK_SMALL_MESH_ELEMS,   // concurrent many-mesh adapt: meshes estimated below this
                         // many elements are adapted together in batch unions
                         // (0: none): 0, 25000, 50000 (default), 100000, 200000
  TK_NKEYS
};
u32 tuned(TuneKey k);
char const* tune_name(u32 k);
// 0, or E_ARG for an unknown name or a value the key does not allow
int tune_set(char const* name, u32 value);
int tune_get(char const* name, u32* value);
// reads a table file; 0, E_IO (unreadable) or E_ARG (a bad line: nothing set)
int tune_load(char const* path);

// thread-local error state behind osh_b200_last_error()
void set_error(int code, char const* msg);
int last_error();
char const* last_error_message();
void clear_error();

// Exclusive scan with the total appended: out has n+1 entries and
// out[n] = sum(in). Single-pass decoupled look-back (uints_exscan, ints.cpp).
// total_to (optional, device): receives out[n] as well (a mailbox slot the
// host reads back with other flags, instead of a copy of its own)
// newid (optional, device, n entries; for 0/1 inputs): out[i] where in[i]
// is 1, INV where 0 -- the new id of each entity the flags mark as kept
void exscan_u32(u32 const* in, u32* out, u32 n, cudaStream_t s, u32* total_to = nullptr,
    u32* newid = nullptr);
u32* exscan_new(u32 const* in, u32 n, cudaStream_t s, u32* total_to = nullptr,
    u32* newid = nullptr);

// Independent scans in one launch (their look-back chains overlap): job j
// scans `in` (mode 0) or the survivors of an offsets array in[0..n]
// (mode 1: in[i + 1] == in[i], uints_negate_offsets) into out[0..n], with
// total_to and newid as above. Jobs are launched MAX_SCAN_JOBS at a time.
constexpr u32 MAX_SCAN_JOBS = 8;
struct ScanJob {
  u32 const* in;
  u32* out;
  u32* total_to;
  u32* newid;
  u32 n;
  u32 mode;
  // (optional, 0/1 items: mode 0 with 0/1 items, or mode 2) list[out[i]] = i
  // where item i is 1: the marked items in order
  u32* list = nullptr;
  // (optional, 0/1 items) the scan of the complement,
  // comp[i] = i - out[i] for i <= n (the unmarked items before i), and
  // comp_newid[i] = comp[i] where item i is 0 and INV where it is 1 -- each
  // survivor's new id when the items mark what a pass removes
  u32* comp = nullptr;
  u32* comp_newid = nullptr;
  // mode 2: item i is 1 where in[i] == stamp, else 0 (marks stamped with a
  // generation, see stream_marks)
  u32 stamp = 0;
};
struct ScanJobs {
  u32 njobs;
  u32 tile0[MAX_SCAN_JOBS + 1];
  ScanJob j[MAX_SCAN_JOBS];
};
void exscan_jobs(ScanJob const* jobs, u32 njobs, cudaStream_t s);

// Scratch kept per (device, stream, key) between calls, zeroed when made or
// grown. stream_zero_scratch: the caller leaves it zero again after each use
// (keys KEPT_ROWS0 and KEPT_ROWS1: the search rows' counts, which the rows'
// fill counts back down to zero). stream_marks: entries stamped with a
// generation of the (stream, key), returned in *gen (never 0) and new on
// every call, so no entry of an earlier use passes for a mark of this one
// (KEPT_MARKS: the products' vertices of a pass's searches; KEPT_FUSED + d:
// the collapses' fused entities of dimension d; KEPT_SPLIT + d: a
// refinement's split domain entities of dimension d).
enum : u32 { KEPT_ROWS0 = 1, KEPT_ROWS1 = 2, KEPT_MARKS = 3, KEPT_FUSED = 4, KEPT_SPLIT = 8 };
u32* stream_zero_scratch(u32 key, size_t words, cudaStream_t s);

// blocks of `block` threads (and `smem` bytes of dynamic shared memory) of a
// kernel resident at once on the current device: the occupancy
// calculator's blocks per SM times the SMs, computed once per kernel, shape
// and device (for grids that stride over their work in one wave)
u32 resident_blocks_of(void const* kernel, u32 block, size_t smem);
template <class K>
inline u32 resident_blocks(K kernel, u32 block, size_t smem = 0)
{
  return resident_blocks_of(reinterpret_cast<void const*>(kernel), block, smem);
}
// frees (in the order of s) the scan and kept scratch of stream s on the
// current device; called before a stream is destroyed, so that scratch does
// not outlive its stream (no kernel may use it afterwards)
void release_stream_scratch(cudaStream_t s);
u32* stream_marks(u32 key, size_t words, cudaStream_t s, u32* gen);

// The same scan with caller-provided scratch of at least
// exscan_scratch_words(n) 32-bit words (zeroed here); allocates nothing.
size_t exscan_scratch_words(u32 n);
void exscan_u32_scratch(u32 const* in, u32* out, u32 n, u32* scratch, cudaStream_t s);

// throws E_TIMEOUT if a bounded device-side wait gave up since the last check
void check_device_timeouts(cudaStream_t s);
// one scan whose second tile waits for a first tile that never publishes,
// with a wait limit of spin_limit polls: E_TIMEOUT when the wait gave up
int selftest_scan_wait(u32 spin_limit);

// out[i] = !(offs[i+1] - offs[i]) scanned (uints_negate_offsets, ints.cpp:227)
// newid (optional): out[i] where entity i is kept, INV where it is not
u32* negate_offsets(u32 const* offs, u32 n, cudaStream_t s, u32* total_to = nullptr,
    u32* newid = nullptr);

void fill_u32(u32* a, u32 n, u32 v, cudaStream_t s);

// grow the device's memory pool to at least `bytes` now (the pool keeps what
// it holds), so that later passes do not pay for growing it
void pool_reserve(unsigned long long bytes);
void pool_stats(unsigned long long* reserved, unsigned long long* used,
    unsigned long long* used_high, int reset_high);
void iota_u32(u32* a, u32 n, u32 stride, cudaStream_t s);
void iota_u64(u64* a, u32 n, cudaStream_t s);

// expand_array (arrays.cpp:170-192): rows of `width` elements of size esz
// copied to every slot [offs[i], offs[i+1]); output rows start at out.
void expand_rows(void const* in, u32 const* offs, u32 n, u32 width, u32 esz,
    void* out, cudaStream_t s);

// max over a u32 array (uints_max)
u32 max_u32(u32 const* a, u32 n, cudaStream_t s);

// Per-kernel event probes. When a probe is enabled, every launch it wraps is
// bracketed by CUDA events on the launching stream and credited with the
// launch's algorithmic bytes (each input read once, each output written
// once); the pairs are resolved after the timed region by probe_read.
enum ProbeId {
  P_REFLECT_DOWN = 0,
  P_UP_COUNT,
  P_UP_FILL,
  P_UP_RANK,
  P_EXSCAN,
  P_ELEM_QUALITY,
  P_REFINE_CANDIDATES,
  P_REFINE_QUALITY,
  P_INDSET_ROUND,
  P_COARSEN_QUALITY,
  P_SWAP_QUALITY,
  P_REFINE_TOPOLOGY,
  P_COLLAPSE_TO_ENT,
  P_EXPAND,
  P_CARRY,
  P_CARRY_UP,
  P_CARRY_UP_FILL,
  P_NPROBES
};
char const* probe_name(u32 id);
// the single-precision filter's device counters (one buffer per device)
struct Fp32Stats;
Fp32Stats* fp32_stats_dev();
void fp32_stats_read(unsigned long long* decided, unsigned long long* rechecked,
    double* max_err, unsigned* bound_exceeded);
void fp32_stats_reset();
// audit mode (every decision taken on an estimate also taken in double) and
// its counters
void fp32_set_audit(bool on);
void fp32_audit_read(unsigned long long* audited, unsigned long long* flips,
    unsigned long long* checked);
// the filter's estimates for n given tets (12 coordinates each) and edges
// (6 coordinates and 2 sizes each), with the double values (filter.cu)
void fp32_probe_tets(u32 n, double const* host_x, float* est, float* err, double* q64);
void fp32_probe_edges(u32 n, double const* host_x, double const* host_h, double thr,
    int* side, double* ratio64);

void probe_enable(u32 mask);
void probe_reset();
void probe_read(u32 id, u32* launches, double* ms, double* bytes);

struct ProbeScope {
  cudaEvent_t a = nullptr, b = nullptr;
  u32 id;
  double bytes;
  cudaStream_t s;
  ProbeScope(u32 id, cudaStream_t s, double bytes);
  ~ProbeScope();
};
#define PROBE(id, stream, bytes) ::osh::ProbeScope osh_probe_scope_((id), (stream), (double)(bytes))

// number of kernels this library launched in the process, and the number of
// times it waited for the device
unsigned long long launch_count();
unsigned long long sync_count();
// device allocations made so far, and host seconds spent waiting in stream
// synchronisations
void host_stats(unsigned long long* allocs, double* sync_seconds);
void stream_sync(cudaStream_t s);
// 64 bytes of pinned host memory owned by the calling host thread, for small
// device-to-host reads (a read into pageable memory is staged by the driver)
void* pinned_scratch();

// small pinned host mailbox for reading several device scalars at once.
// Slots, by the step that writes them (steps of one mesh run one at a time,
// so steps that never overlap share slots):
//   44-50   independent-set rounds: grid barrier, "anything left" flags,
//           rounds run, barrier error (one launch runs every round)
//   1-3     refinement: any good candidate, any inverted child, any candidate
//   4-7     coarsening selection: any collapse kept (4), codes flag (5, not
//           read), listed candidates (7); swap selection: interior
//           candidates (5, not read), any swap kept (6)
//   8-11    refinement build: split entities per domain dimension
//   16-22   coarsening build: products and survivors per dimension, kept
//           vertices (22)
//   20-25   swap build: products and survivors per dimension
//   24-25   classification (derive_model)
//   30-31   size fields (a 64-bit word)
//   60-61   adjacency derivation error flags
// fetch: a one-block kernel stores the slots into the pinned host copy
// (mapped into the device's address space) and then a sequence word, after
// a system-scope fence; the host spins on that word (asking the stream for
// errors as it waits) instead of waiting for a copy and a stream
// synchronisation, which woke the host 6-20 us after the copy ended.
struct Mailbox {
  static constexpr u32 SEQ_SLOT = 64;  // host[SEQ_SLOT]: the last fetch's number
  u32* host = nullptr;   // pinned, 64 slots + the sequence word
  u32* hdev = nullptr;   // host's device address
  u32* dev = nullptr;    // device, 64 slots
  u32 seq = 0;
  void init(cudaStream_t s);
  void release();
  void clear(cudaStream_t s);                 // zero the device slots
  void fetch(cudaStream_t s, u32 nslots = 64);  // the first nslots slots to host
  // nwords (at most 16) 32-bit words of any device array, the same way,
  // into host[READ_SLOT..]; returns that host address
  static constexpr u32 READ_SLOT = SEQ_SLOT + 16;
  u32 const* read(cudaStream_t s, u32 const* src, u32 nwords);
  // nslots words of src into host[at..] and the sequence word after them
  void post(cudaStream_t s, u32 const* src, u32 nslots, u32 at);
};

}  // namespace osh
