// Serving: a request loop over the batched union (batch.hpp) with continuous
// batching. Jobs (a tet mesh and its vertex size field, in host memory) wait
// in a queue until the device-memory budget admits them; an admitted job is
// classified (mesh_derive_model, crease pi/4), joins the running union at the
// next step boundary and takes its own place in mesh_adapt's pass loop; a job
// whose loop ends is split out of the union at that step's end and handed
// back, while the others keep running. Every step is one launch sequence for
// all resident jobs, so jobs that arrive while others run share their passes.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "batch.hpp"
#include "serve.hpp"

namespace osh {

namespace {

double now_s()
{
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// elements an adapted mesh will hold, from the size field: sum over elements
// of volume / (volume of the regular element whose edge is the mean size)
double estimate_elements(u32 dim, u32 nv, double const* x, u32 ne, u32 const* conn,
    double const* h)
{
  double sum = 0;
  u32 vpe = dim + 1;
  // a strided sample of at most 4096 elements, scaled to all of them
  u32 stride = ne > 4096 ? ne / 4096 : 1, taken = 0;
  for (u32 i = 0; i < ne; i += stride) {
    ++taken;
    u32 const* c = conn + (size_t)i * vpe;
    double hm = 0;
    for (u32 j = 0; j < vpe; ++j) hm += h[c[j]];
    hm /= vpe;
    double a[3], b[3], d[3];
    for (u32 k = 0; k < 3; ++k) {
      a[k] = x[c[1] * 3 + k] - x[c[0] * 3 + k];
      b[k] = x[c[2] * 3 + k] - x[c[0] * 3 + k];
      d[k] = dim == 3 ? x[c[3] * 3 + k] - x[c[0] * 3 + k] : 0.0;
    }
    double cr[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
        a[0] * b[1] - a[1] * b[0]};
    double meas, ideal;
    if (dim == 3) {
      meas = std::fabs(cr[0] * d[0] + cr[1] * d[1] + cr[2] * d[2]) / 6.0;
      ideal = hm * hm * hm / (6.0 * std::sqrt(2.0));
    } else {
      meas = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]) / 2.0;
      ideal = hm * hm * std::sqrt(3.0) / 4.0;
    }
    if (ideal > 0) sum += meas / ideal;
  }
  (void)nv;
  return taken ? sum * ((double)ne / taken) : 0.0;
}

}  // namespace

struct ServeJob {
  u32 id = 0;
  u32 dim = 3, nverts = 0, nelems = 0;
  std::vector<double> coords, size;
  std::vector<u32> conn;
  unsigned long long est_bytes = 0;
  Mesh* mesh = nullptr;  // the input before it joins, the result after
  SegState st;
  Layout start;
  double t_submit = 0, t_admit = 0, t_done = 0;
  bool finished = false, taken = false, polled = false;
  ~ServeJob() { delete mesh; }
};

struct Server {
  unsigned long long budget = 0, reserved = 0;
  double t0 = 0;
  GroupRunner run;
  std::map<u32, std::unique_ptr<ServeJob>> jobs;
  std::deque<ServeJob*> queue;
  // resident jobs, each mesh held apart and regrouped per pass
  std::vector<ServeJob*> active;
  std::vector<Mesh*> ms;
  std::vector<SegState> st;
  std::vector<char> owned;
  u32 next_id = 0;
  u32 steps = 0, unions = 0;
  double secs_admit = 0, secs_passes = 0, secs_retire = 0;
  // the engine thread (server_start): it runs steps while there is work;
  // `mu` guards the queue, the job table and the finished flags
  std::mutex mu;
  std::condition_variable cv;
  std::thread engine;
  bool running = false, stopping = false;
  int device = 0;
  int err_code = 0;
  std::string err_msg;

  ~Server()
  {
    stop();
    for (size_t k = 0; k < ms.size(); ++k)
      if (owned[k]) delete ms[k];
    jobs.clear();
    if (run.s) {
      release_stream_scratch(run.s);
      cudaStreamSynchronize(run.s);
      cudaStreamDestroy(run.s);
    }
  }

  void stop()
  {
    {
      std::lock_guard<std::mutex> g(mu);
      if (!running) return;
      stopping = true;
    }
    cv.notify_all();
    engine.join();
    running = false;
    stopping = false;
  }

  void engine_loop()
  {
    cudaSetDevice(device);
    for (;;) {
      {
        std::unique_lock<std::mutex> g(mu);
        cv.wait(g, [&] { return stopping || !queue.empty() || !active.empty(); });
        if (stopping) return;
      }
      try {
        step();
      } catch (Failure const& f) {
        std::lock_guard<std::mutex> g(mu);
        err_code = f.code;
        err_msg = f.what();
        return;
      } catch (std::exception const& e) {
        std::lock_guard<std::mutex> g(mu);
        err_code = E_CUDA;
        err_msg = e.what();
        return;
      }
      cv.notify_all();  // waiters see finished jobs
    }
  }

  void admit()
  {
    cudaStream_t s = run.s;
    for (;;) {
      ServeJob* j = nullptr;
      {
        std::lock_guard<std::mutex> g(mu);
        if (queue.empty()) break;
        j = queue.front();
        if (!active.empty() && reserved + j->est_bytes > budget) break;
        queue.pop_front();
      }
      reserved += j->est_bytes;
      Mesh* m = new Mesh(j->dim, false, false, s);
      try {
        m->set_ents(0, j->nverts, nullptr);
        u32 vpe = deg(j->dim, 0);
        u32* c = dalloc<u32>((size_t)j->nelems * vpe, s);
        CK(cudaMemcpyAsync(c, j->conn.data(), sizeof(u32) * j->conn.size(),
            cudaMemcpyHostToDevice, s));
        m->set_ents(j->dim, j->nelems, c);
        double* x = dalloc<double>((size_t)j->nverts * 3, s);
        CK(cudaMemcpyAsync(x, j->coords.data(), sizeof(double) * j->coords.size(),
            cudaMemcpyHostToDevice, s));
        m->add_tag(0, T_F64, "coordinates", 3, X_NOT, x);
        m->derive_model(3.14159265359 / 4.0);  // PI / 4 with algebra.hpp:8's PI
        double* h = dalloc<double>(j->nverts, s);
        CK(cudaMemcpyAsync(h, j->size.data(), sizeof(double) * j->size.size(),
            cudaMemcpyHostToDevice, s));
        m->add_tag(0, T_F64, "adapt_size", 1, X_POINTWISE, h);
        stream_sync(s);
      } catch (...) {
        delete m;
        throw;
      }
      j->start = layout_of(*m);
      j->t_admit = now_s() - t0;
      // the host copy is no longer needed
      std::vector<double>().swap(j->coords);
      std::vector<double>().swap(j->size);
      std::vector<u32>().swap(j->conn);
      active.push_back(j);
      ms.push_back(m);
      st.push_back(SegState());
      owned.push_back(1);
    }
  }

  u32 step()
  {
    double t_a = now_s();
    admit();
    double t_b = now_s();
    secs_admit += t_b - t_a;
    if (active.empty()) {
      std::lock_guard<std::mutex> g(mu);
      publish();
      return (u32)queue.size();
    }
    steps += 1;
    u32 u0 = last_batch_stats().unions;
    run.step(ms, st, owned);
    check_device_timeouts(run.s);
    unions += last_batch_stats().unions - u0;
    double t_c = now_s();
    secs_passes += t_c - t_b;
    // retire the jobs whose loop ended
    size_t w = 0;
    double t = t_c - t0;
    for (size_t k = 0; k < active.size(); ++k) {
      ServeJob* j = active[k];
      if (st[k].state >= ST_DONE) {
        Mesh* m = ms[k];
        if (!owned[k]) throw Failure(E_ARG, "server lost a job's mesh");
        drop_segments(*m);
        Layout want = j->start;
        for (u32 op : st[k].res.ops) want = layout_after(op, want, m->dim);
        apply_layout(*m, want);
        m->own_new_stream();
        {
          std::lock_guard<std::mutex> g(mu);
          j->st = st[k];
          j->mesh = m;
          j->finished = true;
          j->t_done = t;
        }
        reserved -= j->est_bytes;
        continue;
      }
      active[w] = active[k];
      ms[w] = ms[k];
      st[w] = st[k];
      owned[w] = owned[k];
      ++w;
    }
    active.resize(w);
    ms.resize(w);
    st.resize(w);
    owned.resize(w);
    secs_retire += now_s() - t_c;
    std::lock_guard<std::mutex> g(mu);
    publish();
    return (u32)(active.size() + queue.size());
  }

  // the counters server_stats reports, copied under `mu`
  ServeStats snap;
  void publish()
  {
    snap.steps = steps;
    snap.rebuilds = unions;
    snap.active = (u32)active.size();
    snap.reserved = reserved;
    snap.secs_admit = secs_admit;
    snap.secs_passes = secs_passes;
    snap.secs_retire = secs_retire;
  }
};

Server* server_new(AdaptParams const& ap, unsigned long long budget)
{
  Server* sv = new Server();
  last_batch_stats() = BatchStats();
  sv->run.ap = ap;
  // unions of a few million elements: enough work per launch, and a working
  // set that keeps most gathers in L2
  sv->run.max_union_elems = 4000000ull;
  sv->budget = budget;
  sv->t0 = now_s();
  CK(cudaStreamCreateWithFlags(&sv->run.s, cudaStreamNonBlocking));
  return sv;
}

void server_free(Server* sv) { delete sv; }

u32 server_submit(Server* sv, u32 dim, u32 nverts, double const* coords, u32 nelems,
    u32 const* conn, double const* size)
{
  if (dim < 2 || dim > 3) throw Failure(E_ARG, "jobs are 2D or 3D simplex meshes");
  if (!nverts || !nelems || !coords || !conn || !size) throw Failure(E_ARG, "empty job");
  std::unique_ptr<ServeJob> j(new ServeJob());
  j->dim = dim;
  j->nverts = nverts;
  j->nelems = nelems;
  u32 vpe = dim + 1;
  j->coords.assign(coords, coords + (size_t)nverts * 3);
  j->conn.assign(conn, conn + (size_t)nelems * vpe);
  j->size.assign(size, size + nverts);
  for (u32 c : j->conn)
    if (c >= nverts) throw Failure(E_ARG, "job connectivity names a missing vertex");
  double est = estimate_elements(dim, nverts, coords, nelems, conn, size);
  if (est < nelems) est = nelems;
  // device bytes per element while a mesh adapts (connectivity of every
  // dimension, the adjacency a pass derives, and the next mesh being built)
  j->est_bytes = (unsigned long long)(est * 900.0);
  u32 id;
  {
    std::lock_guard<std::mutex> g(sv->mu);
    j->id = sv->next_id++;
    j->t_submit = now_s() - sv->t0;
    sv->queue.push_back(j.get());
    id = j->id;
    sv->jobs[id] = std::move(j);
  }
  sv->cv.notify_all();
  return id;
}

u32 server_step(Server* sv)
{
  if (sv->running) throw Failure(E_ARG, "the server's engine thread runs its steps");
  return sv->step();
}

void server_start(Server* sv)
{
  std::lock_guard<std::mutex> g(sv->mu);
  if (sv->running) return;
  CK(cudaGetDevice(&sv->device));
  sv->running = true;
  sv->engine = std::thread([sv] { sv->engine_loop(); });
}

void server_stop(Server* sv) { sv->stop(); }

int server_wait(Server* sv, double timeout_s)
{
  std::unique_lock<std::mutex> g(sv->mu);
  auto pending = [&] {
    u32 n = (u32)sv->queue.size();
    for (auto const& kv : sv->jobs)
      if (!kv.second->finished && std::find(sv->queue.begin(), sv->queue.end(),
                                              kv.second.get()) == sv->queue.end())
        ++n;
    return n;
  };
  auto done = [&] { return sv->err_code != 0 || pending() == 0; };
  if (timeout_s < 0)
    sv->cv.wait(g, done);
  else
    sv->cv.wait_for(g, std::chrono::duration<double>(timeout_s), done);
  if (sv->err_code) throw Failure(sv->err_code, sv->err_msg);
  return (int)pending();
}

void server_set_union_elems(Server* sv, unsigned long long n) { sv->run.max_union_elems = n; }

std::vector<u32> server_poll(Server* sv, u32 max_ids)
{
  std::lock_guard<std::mutex> g(sv->mu);
  std::vector<u32> out;
  for (auto& kv : sv->jobs)
    if (kv.second->finished && !kv.second->polled && out.size() < max_ids) {
      kv.second->polled = true;
      out.push_back(kv.first);
    }
  return out;
}

Mesh* server_take(Server* sv, u32 id)
{
  std::lock_guard<std::mutex> g(sv->mu);
  auto it = sv->jobs.find(id);
  if (it == sv->jobs.end() || !it->second->finished || it->second->taken)
    throw Failure(E_ARG, "no finished job with that id to take");
  Mesh* m = it->second->mesh;
  it->second->mesh = nullptr;
  it->second->taken = true;
  return m;
}

ServeJobInfo server_job_info(Server* sv, u32 id)
{
  std::lock_guard<std::mutex> g(sv->mu);
  auto it = sv->jobs.find(id);
  if (it == sv->jobs.end()) throw Failure(E_ARG, "no job with that id");
  ServeJob const& j = *it->second;
  ServeJobInfo r;
  r.t_submit = j.t_submit;
  r.t_admit = j.t_admit;
  r.t_done = j.t_done;
  r.finished = j.finished;
  r.passes = j.st.res.passes;
  r.elems_in = j.st.res.elems_in;
  r.status = j.st.res.status;
  r.changed = j.st.res.changed;
  return r;
}

ServeStats server_stats(Server* sv)
{
  std::lock_guard<std::mutex> g(sv->mu);
  ServeStats r = sv->snap;
  r.queued = (u32)sv->queue.size();
  r.now = now_s() - sv->t0;
  return r;
}

}  // namespace osh
