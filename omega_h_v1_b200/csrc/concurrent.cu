// Many meshes adapted concurrently: mesh_adapt (adapt.cpp:82-94) of each
// mesh, unchanged, run by a few host threads, each issuing on a CUDA stream
// of its own, so that the passes of different meshes overlap on the device.
// One mesh's passes leave the GPU idle while the host reads a count back or
// launches its next kernel; another mesh's kernels fill those gaps, and small
// meshes, whose passes are all latency, run side by side. Each mesh is
// adapted by exactly the code osh_adapt runs, so it ends exactly as osh_adapt
// leaves it.
//
// Memory: a mesh is started only while the device-memory estimates of the
// meshes in flight (elements the size field asks for, or the current count
// if larger, times 900 bytes) fit a budget; meshes start largest first, and
// a mesh larger than the budget runs alone.
#include <algorithm>
#include <condition_variable>
#include <mutex>
#include <thread>

#include "batch.hpp"

namespace osh {

namespace {

// elements the mesh will hold after adaptation, from its size field: the
// sum over elements of volume / (volume of the regular element whose edge
// is the element's mean size)
__global__ void k_estimate_elements(u32 dim, u32 ne, u32 const* __restrict__ voe,
    double const* __restrict__ x, double const* __restrict__ h, double* out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  double r = 0;
  if (i < ne) {
    u32 vpe = dim + 1;
    u32 const* c = voe + (size_t)i * vpe;
    double hm = 0;
    for (u32 j = 0; j < vpe; ++j) hm += h[c[j]];
    hm /= vpe;
    double a[3], b[3], d[3] = {0, 0, 0};
    for (u32 k = 0; k < 3; ++k) {
      a[k] = x[c[1] * 3 + k] - x[c[0] * 3 + k];
      b[k] = x[c[2] * 3 + k] - x[c[0] * 3 + k];
      if (dim == 3) d[k] = x[c[3] * 3 + k] - x[c[0] * 3 + k];
    }
    double cr0 = a[1] * b[2] - a[2] * b[1], cr1 = a[2] * b[0] - a[0] * b[2],
           cr2 = a[0] * b[1] - a[1] * b[0];
    double meas, ideal;
    if (dim == 3) {
      meas = fabs(cr0 * d[0] + cr1 * d[1] + cr2 * d[2]) / 6.0;
      ideal = hm * hm * hm / (6.0 * sqrt(2.0));
    } else {
      meas = sqrt(cr0 * cr0 + cr1 * cr1 + cr2 * cr2) / 2.0;
      ideal = hm * hm * sqrt(3.0) / 4.0;
    }
    r = ideal > 0 ? meas / ideal : 0.0;
  }
  for (int o = 16; o; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  if ((threadIdx.x & 31) == 0 && r != 0) atomicAdd(out, r);
}

constexpr double BYTES_PER_ELEMENT = 900.0;  // as the server's admission
// a group of small meshes: at most this many estimated elements, adapted in
// unions of at most SMALL_UNION_ELEMS current elements
constexpr double SMALL_GROUP_ELEMS = 4.0e6;
constexpr unsigned long long SMALL_UNION_ELEMS = 1000000ull;

unsigned long long estimate_bytes(Mesh& m)
{
  u32 ne = m.count(m.dim);
  double est = ne;
  Tag* h = m.find_tag(0, "adapt_size");
  if (h && ne && m.dim >= 2) {
    double* sum = dalloc<double>(1, m.s);
    CK(cudaMemsetAsync(sum, 0, sizeof(double), m.s));
    CK(launch_kernel(k_estimate_elements, dim3(grid_for(ne)), dim3(BLOCK), 0, m.s, m.dim, ne, m.ask_down(m.dim, 0),
        m.coords(), static_cast<double const*>(h->data), sum));
    CK_LAUNCH();
    est = std::max(est, read_f64(sum, m.s));
    dev_free(sum, m.s);
  }
  return (unsigned long long)(est * BYTES_PER_ELEMENT);
}

}  // namespace

void adapt_concurrent(std::vector<Mesh*> const& ms, AdaptParams const& ap, u32 nthreads,
    unsigned long long budget, std::vector<BatchMeshResult>& res)
{
  u32 n = (u32)ms.size();
  res.assign(n, BatchMeshResult());
  if (!n) return;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (!nthreads) nthreads = 4;
  nthreads = std::min(nthreads, n);
  if (!budget) {
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    budget = (unsigned long long)(0.7 * (double)fr);
  }
  std::vector<unsigned long long> est(n);
  for (u32 i = 0; i < n; ++i) est[i] = estimate_bytes(*ms[i]);
  std::vector<u32> order(n);
  for (u32 i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
      [&](u32 a, u32 b) { return est[a] > est[b]; });
  // Work items, largest first: a large mesh is an item of its own; meshes
  // estimated below the tuning table's small_mesh_elems, whose passes are
  // all launch latency, are grouped (up to SMALL_GROUP_ELEMS estimated
  // elements a group, each group batchable: same dimension, entities and
  // tags) and adapted together by adapt_batch, one launch per stage for the
  // group. Every mesh still ends exactly as osh_adapt leaves it.
  std::vector<std::vector<u32>> items;
  std::vector<unsigned long long> item_est;
  {
    double const small = tuned(TK_SMALL_MESH_ELEMS);
    double const cap = SMALL_GROUP_ELEMS;
    std::vector<u32> group;
    double group_elems = 0;
    auto close_group = [&]() {
      if (group.empty()) return;
      unsigned long long e = 0;
      for (u32 k : group) e += est[k];
      items.push_back(group);
      item_est.push_back(e);
      group.clear();
      group_elems = 0;
    };
    for (u32 k : order) {
      double elems = (double)est[k] / BYTES_PER_ELEMENT;
      bool fits = elems < small;
      if (fits && !group.empty()) {
        try {
          check_batchable({ms[group[0]], ms[k]});
        } catch (Failure const&) {
          fits = false;
        }
      } else if (fits) {
        try {
          check_batchable({ms[k]});
        } catch (Failure const&) {
          fits = false;
        }
      }
      if (!fits) {
        items.push_back({k});
        item_est.push_back(est[k]);
        continue;
      }
      if (group_elems + elems > cap) close_group();
      group.push_back(k);
      group_elems += elems;
    }
    close_group();
  }
  u32 const nitems = (u32)items.size();
  nthreads = std::min(nthreads, nitems);
  // a mailbox shared by two of the meshes is replaced for the call: their
  // passes would otherwise read back each other's flags
  std::vector<std::shared_ptr<Mailbox>> saved_mb(n);
  {
    std::vector<Mailbox*> seen;
    for (u32 i = 0; i < n; ++i) {
      Mailbox* p = ms[i]->mb.get();
      if (std::find(seen.begin(), seen.end(), p) != seen.end()) {
        saved_mb[i] = ms[i]->mb;
        ms[i]->mb = std::shared_ptr<Mailbox>(new Mailbox(), [](Mailbox* q) {
          q->release();
          delete q;
        });
        ms[i]->mb->init(ms[i]->s);
      } else {
        seen.push_back(p);
      }
    }
    for (u32 i = 0; i < n; ++i) stream_sync(ms[i]->s);
  }
  std::mutex mu;
  std::condition_variable cv;
  u32 next = 0;
  unsigned long long inflight = 0;
  int first_error = 0;
  std::string first_msg;
  auto worker = [&]() {
    cudaStream_t st = nullptr;
    try {
      CK(cudaSetDevice(dev));
      CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    } catch (Failure const& f) {
      std::lock_guard<std::mutex> g(mu);
      if (!first_error) {
        first_error = f.code;
        first_msg = f.what();
      }
      return;
    }
    for (;;) {
      u32 it;
      {
        std::unique_lock<std::mutex> g(mu);
        cv.wait(g, [&]() {
          return next >= nitems || inflight == 0 || inflight + item_est[next] <= budget;
        });
        if (next >= nitems) break;
        it = next++;
        inflight += item_est[it];
      }
      if (items[it].size() > 1) {
        // a group of small meshes through the batched path
        std::vector<Mesh*> gm;
        std::vector<cudaStream_t> orig;
        for (u32 k : items[it]) {
          gm.push_back(ms[k]);
          orig.push_back(ms[k]->s);
          if (!ms[k]->own_stream) ms[k]->s = st;
        }
        std::vector<BatchMeshResult> gr;
        try {
          adapt_batch(gm, ap.size_floor, ap.good_qual, ap.nlayers, ap.max_ops,
              SMALL_UNION_ELEMS, gr);
          for (size_t j = 0; j < gm.size(); ++j) res[items[it][j]] = gr[j];
        } catch (Failure const& f) {
          std::lock_guard<std::mutex> g(mu);
          if (!first_error) {
            first_error = f.code;
            first_msg = f.what();
          }
        } catch (std::exception const& e) {
          std::lock_guard<std::mutex> g(mu);
          if (!first_error) {
            first_error = E_CUDA;
            first_msg = e.what();
          }
        }
        for (size_t j = 0; j < gm.size(); ++j) {
          cudaStreamSynchronize(gm[j]->s);
          gm[j]->s = orig[j];
        }
        {
          std::lock_guard<std::mutex> g(mu);
          inflight -= item_est[it];
        }
        cv.notify_all();
        continue;
      }
      u32 const k = items[it][0];
      Mesh& m = *ms[k];
      // a mesh on a stream of its own keeps it; one on a stream it may share
      // (the legacy default stream, a caller's stream) runs on the worker's
      cudaStream_t orig = m.s;
      if (!m.own_stream) m.s = st;
      BatchMeshResult& r = res[k];
      try {
        r.changed = mesh_adapt(m, ap.size_floor, ap.good_qual, ap.nlayers, ap.max_ops);
      } catch (Failure const& f) {
        if (f.code == E_MAXOPS) {
          r.status = E_MAXOPS;
        } else {
          std::lock_guard<std::mutex> g(mu);
          if (!first_error) {
            first_error = f.code;
            first_msg = f.what();
          }
        }
      } catch (std::exception const& e) {
        std::lock_guard<std::mutex> g(mu);
        if (!first_error) {
          first_error = E_CUDA;
          first_msg = e.what();
        }
      }
      r.passes = last_adapt_stats().passes;
      r.elems_in = last_adapt_stats().elems_in;
      cudaStreamSynchronize(m.s);
      m.s = orig;
      {
        std::lock_guard<std::mutex> g(mu);
        inflight -= item_est[it];
      }
      cv.notify_all();
    }
    release_stream_scratch(st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  };
  std::vector<std::thread> th;
  for (u32 t = 0; t < nthreads; ++t) th.emplace_back(worker);
  for (auto& t : th) t.join();
  for (u32 i = 0; i < n; ++i)
    if (saved_mb[i]) ms[i]->mb = saved_mb[i];
  BatchStats& bs = last_batch_stats();
  bs = BatchStats();
  for (u32 i = 0; i < n; ++i) {
    bs.mesh_passes += res[i].passes;
    bs.elems_in += res[i].elems_in;
  }
  if (first_error) throw Failure(first_error, first_msg);
}

}  // namespace osh
