// Upward adjacency for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc (or any allocator) at the point where
// they need an upward adjacency: code that runs while a CUDA stream is being
// captured into a graph (an allocation there breaks or invalidates the
// capture), code inside a host callback or a real-time loop that must not
// block on the allocator, and host codes (mesh databases, solvers) that hand
// the GPU a fixed memory budget and own every byte of it. This entry point
// serves them: the caller passes the input and the three output arrays, and
// the scratch the derivation needs (per-row counts, the unsorted rows and
// the scan's tile status) lives in one fixed array in device memory that is
// part of the library image.
#include "../../include/omega_h_b200.h"
#include "mesh.hpp"

namespace osh {

// Scratch for osh_b200_up_from_down_noalloc. Sized for the stated maxima
// OSH_B200_NOALLOC_MAX_USES and OSH_B200_NOALLOC_MAX_LOWS; every GPU that
// loads the library holds it until the process exits.
// (regions padded to 256-byte boundaries: two pads of at most 63 words)
constexpr size_t NOALLOC_SCRATCH_WORDS =
    ((size_t)OSH_B200_NOALLOC_MAX_LOWS + 1) + (size_t)OSH_B200_NOALLOC_MAX_USES +
    (4 + 2 * (((size_t)OSH_B200_NOALLOC_MAX_LOWS + 2047) / 2048)) + 128;

static __device__ __align__(256) u32 noalloc_scratch[NOALLOC_SCRATCH_WORDS];

// In host code `noalloc_scratch` names a host-side stand-in, not device
// memory; its device address is looked up once per device, with that device
// current.
static u32* scratch_address()
{
  static u32* addr[64] = {};
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw Failure(E_ARG, "device ordinal above 63");
  if (!addr[dev]) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, noalloc_scratch));
    addr[dev] = static_cast<u32*>(p);
  }
  return addr[dev];
}

}  // namespace osh

extern "C" int osh_b200_up_from_down_noalloc(unsigned high_dim, unsigned low_dim,
    unsigned nhighs, unsigned nlows, unsigned const* lows_of_highs, unsigned* offsets,
    unsigned* highs_of_lows, unsigned* directions, void* stream)
{
  try {
    if (low_dim >= high_dim || high_dim > 3)
      throw osh::Failure(osh::E_ARG, "up_from_down_noalloc: need low_dim < high_dim <= 3");
    unsigned long long nuses = (unsigned long long)nhighs * osh::deg(high_dim, low_dim);
    if (nuses > OSH_B200_NOALLOC_MAX_USES)
      throw osh::Failure(osh::E_ARG,
          "up_from_down_noalloc: nhighs * deg(high,low) exceeds OSH_B200_NOALLOC_MAX_USES");
    if (nlows > OSH_B200_NOALLOC_MAX_LOWS)
      throw osh::Failure(osh::E_ARG,
          "up_from_down_noalloc: nlows exceeds OSH_B200_NOALLOC_MAX_LOWS");
    if (!offsets || (nuses && (!lows_of_highs || !highs_of_lows || !directions)))
      throw osh::Failure(osh::E_ARG, "up_from_down_noalloc: null array");
    if (osh::up_from_down_scratch_words((osh::u32)nuses, nlows) > osh::NOALLOC_SCRATCH_WORDS)
      throw osh::Failure(osh::E_ARG, "up_from_down_noalloc: scratch too small");
    osh::UpAdj out;
    out.offs = offsets;
    out.adj = highs_of_lows;
    out.dirs = directions;
    osh::up_from_down_scratch(high_dim, low_dim, nhighs, nlows, lows_of_highs, out,
        osh::scratch_address(), static_cast<cudaStream_t>(stream));
    return 0;
  } catch (osh::Failure const& f) {
    osh::set_error(f.code, f.what());
    return f.code;
  } catch (std::exception const& e) {
    osh::set_error(osh::E_CUDA, e.what());
    return osh::E_CUDA;
  }
}
