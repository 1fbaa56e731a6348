// Serving loop with continuous batching over the batched union (serve.cu).
#pragma once

#include <vector>

#include "batch.hpp"

namespace osh {

struct Server;

struct ServeJobInfo {
  double t_submit = 0, t_admit = 0, t_done = 0;  // seconds since server_new
  bool finished = false;
  u32 passes = 0;
  double elems_in = 0;
  int status = 0;
  u32 changed = 0;
};

struct ServeStats {
  u32 steps = 0, rebuilds = 0, active = 0, queued = 0;  // rebuilds: unions formed
  unsigned long long reserved = 0;  // estimated device bytes of resident jobs
  double now = 0;
  // host wall time spent admitting (upload + classification), joining jobs to
  // the running union, in passes, and retiring finished jobs
  double secs_admit = 0, secs_join = 0, secs_passes = 0, secs_retire = 0;
};

Server* server_new(AdaptParams const& ap, unsigned long long budget_bytes);
void server_free(Server* sv);
// queue a job (host arrays are copied); returns its id
u32 server_submit(Server* sv, u32 dim, u32 nverts, double const* coords, u32 nelems,
    u32 const* conn, double const* size);
// admit what the budget allows, run one step over every resident job, hand
// back the jobs whose loop ended; returns the jobs still queued or running
u32 server_step(Server* sv);
// run steps on an engine thread of the server's own (submissions then
// overlap the GPU work); server_wait blocks until every submitted job has
// finished or timeout_s passes (< 0: no limit) and returns the jobs left
void server_start(Server* sv);
void server_stop(Server* sv);
int server_wait(Server* sv, double timeout_s);
// largest union a pass forms, in current elements (0 = no limit)
void server_set_union_elems(Server* sv, unsigned long long n);
// finished jobs not yet reported, at most max_ids of them
std::vector<u32> server_poll(Server* sv, u32 max_ids);
Mesh* server_take(Server* sv, u32 id);
ServeJobInfo server_job_info(Server* sv, u32 id);
ServeStats server_stats(Server* sv);

}  // namespace osh
