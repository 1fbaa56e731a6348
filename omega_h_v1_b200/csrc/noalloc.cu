// Upward adjacency for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc (or any allocator) at the point where
// they need an upward adjacency: code inside a host callback or a real-time
// loop that must not block on the allocator or the driver's memory
// bookkeeping, and host codes (mesh databases, solvers) that hand the GPU a
// fixed memory budget and own every byte of it. This entry point serves
// them: the caller passes the input and the three output arrays, and the
// scratch the derivation needs (a status word, per-row counts, the unsorted
// rows and the scan's tile status) lives in one fixed array in device
// memory that is part of the library image.
//
// The kernels here check what they index: an entry of lows_of_highs that is
// not below nlows, or a scan whose bounded wait gave up, sets the status
// word, after which no kernel of the call writes through a computed index,
// and the last kernel writes 0xffffffff to offsets[nlows] (whose value is
// nuses when the call succeeded).
#include <mutex>

#include "../../include/omega_h_b200.h"
#include "mesh.hpp"

namespace osh {

namespace {

// word offsets of the scratch regions, each on a 256-byte boundary (the
// scan's tile status is read and written as 64-bit words)
constexpr size_t align64w(size_t w) { return (w + 63) & ~(size_t)63; }
constexpr size_t NA_STATUS = 0;   // word 0: error bits of the call
constexpr size_t NA_COUNTS = 64;  // nlows + 1 per-row counts
constexpr size_t na_rows_at(size_t nlows) { return align64w(NA_COUNTS + nlows + 1); }
constexpr size_t na_scan_at(size_t nuses, size_t nlows) { return align64w(na_rows_at(nlows) + nuses); }
// the scan needs 4 + 2 * ceil(n / tile) words with 8192-element tiles; the
// bound below assumes tiles of 2048 and so covers it
constexpr size_t na_words_bound(size_t nuses, size_t nlows)
{
  return na_scan_at(nuses, nlows) + 4 + 2 * ((nlows + 2047) / 2048);
}

constexpr u32 NA_BAD_INPUT = 1u;  // an entry of lows_of_highs >= nlows
constexpr u32 NA_SCAN_WAIT = 2u;  // the scan's bounded look-back gave up
constexpr u32 NA_BAD_SLOT = 4u;   // a row slot fell outside the uses

}  // namespace

// Scratch for osh_b200_up_from_down_noalloc, sized for the stated maxima
// OSH_B200_NOALLOC_MAX_USES and OSH_B200_NOALLOC_MAX_LOWS (about 8.4 MB);
// every GPU that loads the library holds it until the process exits.
constexpr size_t NOALLOC_SCRATCH_WORDS =
    na_words_bound(OSH_B200_NOALLOC_MAX_USES, OSH_B200_NOALLOC_MAX_LOWS);

static __device__ __align__(256) u32 noalloc_scratch[NOALLOC_SCRATCH_WORDS];

namespace {

// In host code `noalloc_scratch` names a host-side stand-in, not device
// memory; its device address is looked up once per device, with that device
// current, the first time a call runs there.
std::once_flag g_addr_once[64];
u32* g_addr[64] = {};

u32* scratch_address()
{
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw Failure(E_ARG, "device ordinal above 63");
  std::call_once(g_addr_once[dev], [dev]() {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, noalloc_scratch));
    g_addr[dev] = static_cast<u32*>(p);
  });
  if (!g_addr[dev]) throw Failure(E_CUDA, "up_from_down_noalloc: scratch address unknown");
  return g_addr[dev];
}

// per-row counts; an out-of-range entry is reported, never used as an index
__global__ void k_na_count(u32 const* __restrict__ loh, u32 nuses, u32 nlows,
    u32* __restrict__ cnt, u32* status)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nuses) return;
  u32 l = loh[i];
  if (l < nlows)
    atomicAdd(&cnt[l], 1u);
  else
    atomicOr(status, NA_BAD_INPUT);
}

// each use placed in its row, from the row's end down (rows are ranked
// afterwards); nothing is written once the status or the scan reports a
// failure, and every slot is checked against the uses
__global__ void k_na_fill(u32 const* __restrict__ loh, u32 nuses, u32 nlows,
    u32 const* __restrict__ offs, u32* __restrict__ cnt, u32* __restrict__ rows,
    u32* status, u32 const* scan_err)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nuses) return;
  if (*(volatile u32*)status || *(volatile u32 const*)scan_err) {
    if (i == 0 && *(volatile u32 const*)scan_err) atomicOr(status, NA_SCAN_WAIT);
    return;
  }
  u32 l = loh[i];
  if (l >= nlows) return;
  u32 slot = offs[l] + atomicSub(&cnt[l], 1u) - 1u;
  if (slot >= offs[l] && slot < offs[l + 1] && offs[l + 1] <= nuses)
    rows[slot] = i;
  else
    atomicOr(status, NA_BAD_SLOT);
}

// one warp per row: each lane ranks its use against the whole row and
// writes it to its sorted place (uses in a row are distinct)
__global__ void k_na_rank(u32 const* __restrict__ offs, u32 const* __restrict__ rows,
    u32 nrows, u32 nuses, u32 lph, u32* __restrict__ adj, u32* __restrict__ dirs,
    u32 const* status)
{
  pdl_wait();
  u32 row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  u32 lane = threadIdx.x & 31;
  if (row >= nrows || *(volatile u32 const*)status) return;
  u32 f = offs[row], e = offs[row + 1];
  if (f > e || e > nuses) return;  // only after a failure, which the status holds
  u32 len = e - f;
  for (u32 base = 0; base < len; base += 32) {
    u32 idx = base + lane;
    u32 my = idx < len ? rows[f + idx] : INV;
    u32 rank = 0;
    for (u32 cb = 0; cb < len; cb += 32) {
      u32 other = (cb + lane < len) ? rows[f + cb + lane] : INV;
      u32 lim = len - cb < 32 ? len - cb : 32;
      for (u32 j = 0; j < lim; ++j) {
        u32 v = __shfl_sync(0xffffffffu, other, j);
        rank += (v < my) ? 1u : 0u;
      }
    }
    if (idx < len && rank < len) {
      adj[f + rank] = my / lph;
      dirs[f + rank] = my % lph;
    }
  }
}

// a failed call says so in offsets[nlows], whose value is nuses otherwise
__global__ void k_na_finish(u32 nlows, u32* offs, u32 const* status, u32 const* scan_err)
{
  pdl_wait();
  if (*(volatile u32 const*)status || *(volatile u32 const*)scan_err) offs[nlows] = INV;
}

}  // namespace

}  // namespace osh

extern "C" int osh_b200_up_from_down_noalloc(unsigned high_dim, unsigned low_dim,
    unsigned nhighs, unsigned nlows, unsigned const* lows_of_highs, unsigned* offsets,
    unsigned* highs_of_lows, unsigned* directions, void* stream)
{
  using namespace osh;
  try {
    if (low_dim >= high_dim || high_dim > 3)
      throw Failure(E_ARG, "up_from_down_noalloc: need low_dim < high_dim <= 3");
    u32 const lph = deg(high_dim, low_dim);
    unsigned long long nuses = (unsigned long long)nhighs * lph;
    if (nuses > OSH_B200_NOALLOC_MAX_USES)
      throw Failure(E_ARG,
          "up_from_down_noalloc: nhighs * deg(high,low) exceeds OSH_B200_NOALLOC_MAX_USES");
    if (nlows > OSH_B200_NOALLOC_MAX_LOWS)
      throw Failure(E_ARG, "up_from_down_noalloc: nlows exceeds OSH_B200_NOALLOC_MAX_LOWS");
    if (!offsets || (nuses && (!lows_of_highs || !highs_of_lows || !directions)))
      throw Failure(E_ARG, "up_from_down_noalloc: null array");
    size_t const scan_at = na_scan_at(nuses, nlows);
    if (scan_at + exscan_scratch_words(nlows) > NOALLOC_SCRATCH_WORDS)
      throw Failure(E_ARG, "up_from_down_noalloc: scratch too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    u32* scratch = scratch_address();
    u32* status = scratch + NA_STATUS;
    u32* cnt = scratch + NA_COUNTS;
    u32* rows = scratch + na_rows_at(nlows);
    u32* scan = scratch + scan_at;
    // the status word and the counts are contiguous: one clear for both
    CK(cudaMemsetAsync(scratch, 0, sizeof(u32) * (NA_COUNTS + (size_t)nlows + 1), s));
    u32 const n = (u32)nuses;
    if (n) {
      CK(launch_kernel(k_na_count, dim3(grid_for(n)), dim3(BLOCK), 0, s, lows_of_highs, n, nlows, cnt, status));
      CK_LAUNCH();
    }
    // clears its own scratch (word 1 of which records a wait that gave up)
    exscan_u32_scratch(cnt, offsets, nlows, scan, s);
    if (n) {
      CK(launch_kernel(k_na_fill, dim3(grid_for(n)), dim3(BLOCK), 0, s, lows_of_highs, n, nlows, offsets, cnt, rows,
          status, scan + 1));
      CK_LAUNCH();
      u64 threads = (u64)nlows * 32;
      CK(launch_kernel(k_na_rank, dim3(grid_for(threads)), dim3(BLOCK), 0, s, offsets, rows, nlows, n, lph,
          highs_of_lows, directions, status));
      CK_LAUNCH();
    }
    CK(launch_kernel(k_na_finish, dim3(1), dim3(1), 0, s, nlows, offsets, status, scan + 1));
    CK_LAUNCH();
    return 0;
  } catch (Failure const& f) {
    set_error(f.code, f.what());
    return f.code;
  } catch (std::exception const& e) {
    set_error(E_CUDA, e.what());
    return E_CUDA;
  }
}
