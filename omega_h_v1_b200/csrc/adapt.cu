// mesh_adapt (adapt.cpp:36-94): refine until nothing splits, coarsen until
// nothing collapses, then fix slivers by swapping (3D) or collapsing, with a
// cap on the number of passes.
#include <cstdio>
#include <cstdlib>

#include "passes.hpp"

namespace osh {

static bool verbose()
{
  static int v = -1;
  if (v < 0) {
    char const* e = std::getenv("OSH_B200_VERBOSE");
    v = (e && *e && *e != '0') ? 1 : 0;
  }
  return v == 1;
}

static void report(Mesh& m, char const* what)
{
  if (!verbose()) return;
  PassStats const& st = last_pass_stats();
  std::printf("%s: %u selected, %u -> %u elements, %u independent-set rounds\n", what,
      st.nselected, st.elems_in, st.elems_out, st.indset_rounds);
  (void)m;
}

AdaptStats& last_adapt_stats()
{
  static thread_local AdaptStats s;
  return s;
}

u32 mesh_adapt(Mesh& m, double size_floor, double good_qual, u32 nlayers, u32 max_ops)
{
  u32 ops = 0;
  AdaptStats& as = last_adapt_stats();
  as = AdaptStats();
  auto incr = [&](char const* what) {
    as.passes += 1;
    as.elems_in += last_pass_stats().elems_in;
    // incr_op_count (adapt.cpp:36-45) aborts; this build reports E_MAXOPS
    if (ops > max_ops) throw Failure(E_MAXOPS, "mesh_adapt exceeded max_passes");
    ++ops;
    report(m, what);
  };
  double qf = m.min_quality();
  if (good_qual < qf) qf = good_qual;
  while (refine_by_size(m, qf)) incr("refine");
  while (coarsen_by_size(m, qf, size_floor)) incr("coarsen");
  for (;;) {
    double prev = m.min_quality();
    if (prev >= good_qual) break;
    if (m.dim == 3 && swap_slivers(m, good_qual, nlayers)) {
      incr("swap");
      continue;
    }
    if (coarsen_slivers(m, good_qual, nlayers)) {
      incr("coarsen slivers");
      continue;
    }
    if (verbose()) std::printf("warning: shape quality could not be satisfied\n");
    break;
  }
  return ops > 0;
}

}  // namespace osh
