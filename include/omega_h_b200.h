/*
 * omega_h_b200.h -- entry points of libosh_b200.so beyond the public
 * omega_h.h. They expose the reference's internal C++ entry points for the
 * adaptation pass (C linkage here) plus the helpers a caller needs with a
 * device-resident mesh. All mesh arrays are device memory; arguments named
 * host_* are host memory.
 */
#ifndef OMEGA_H_B200_H
#define OMEGA_H_B200_H

#include <stddef.h>

#include "omega_h.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error reporting (the reference asserts / aborts instead) ---------- */
enum osh_b200_error {
  OSH_B200_OK = 0,
  OSH_B200_E_CUDA = 1,
  OSH_B200_E_NOCONVERGE = 2, /* independent set not settled in 100 rounds */
  OSH_B200_E_MAXOPS = 3,     /* mesh_adapt exceeded max_passes */
  OSH_B200_E_ARG = 4,
  OSH_B200_E_NOMEM = 5,
  OSH_B200_E_UNSUPPORTED = 6,
  OSH_B200_E_TIMEOUT = 7,
  OSH_B200_E_INVERTED = 8,
  OSH_B200_E_IO = 9          /* a mesh file could not be opened, read or parsed */
};
int osh_b200_last_error(void) OSH_PUBLIC;
char const* osh_b200_last_error_message(void) OSH_PUBLIC;
void osh_b200_clear_error(void) OSH_PUBLIC;

/* ---- the adaptation passes (reference C++ entry points) ---------------- */
/* refine_by_size (refine.hpp:8, refine.cpp:17-27) */
unsigned osh_b200_refine_by_size(osh_t m, double qual_floor) OSH_PUBLIC;
/* uniformly_refine (refine.hpp:9, refine.cpp:29-35) */
void osh_b200_uniformly_refine(osh_t m) OSH_PUBLIC;
/* coarsen_by_size (coarsen.hpp:8-11, coarsen.cpp:23-36) */
unsigned osh_b200_coarsen_by_size(osh_t m, double qual_floor,
    double size_ratio_floor) OSH_PUBLIC;
/* coarsen_slivers (coarsen.hpp:13-16, coarsen.cpp:51-70) */
unsigned osh_b200_coarsen_slivers(osh_t m, double qual_floor,
    unsigned nlayers) OSH_PUBLIC;
/* swap_slivers (swap.hpp:8-11, swap.cpp:138-154) */
unsigned osh_b200_swap_slivers(osh_t m, double good_qual,
    unsigned nlayers) OSH_PUBLIC;
/* mesh_adapt (adapt.hpp:8-12, adapt.cpp:82-94); same as osh_adapt */
unsigned osh_b200_mesh_adapt(osh_t m, double size_ratio_floor,
    double good_qual, unsigned nsliver_layers, unsigned max_passes) OSH_PUBLIC;
/* mesh_min_quality (quality.cpp:67-73), minimum over every element */
double osh_b200_min_quality(osh_t m) OSH_PUBLIC;

/* statistics of the last pass run on this thread: op (1 refine, 2 coarsen,
   3 swap, 4 coarsen slivers), elements in / out, selected entities and
   independent-set rounds */
void osh_b200_last_pass(unsigned* op, unsigned* elems_in, unsigned* elems_out,
    unsigned* nselected, unsigned* rounds) OSH_PUBLIC;

/* ---- many meshes adapted together --------------------------------------- */
/* No single counterpart in the reference: mesh_adapt (adapt.cpp:82-94) of
   every mesh in `meshes`, with the meshes concatenated into disjoint unions
   of at most max_union_elems input elements (0 = one union) so that each
   stage of a pass is one launch for all of them. Each mesh ends exactly as
   osh_adapt would leave it; meshes that changed are replaced in place.
   changed[i] (optional) receives what osh_adapt would return for mesh i and
   status[i] (optional) 0 or OSH_B200_E_MAXOPS. All meshes must have the same
   dimension, representation and tags. Returns 0 or an error code. */
int osh_b200_adapt_batch(osh_t* meshes, unsigned nmeshes, double size_ratio_floor,
    double good_qual, unsigned nsliver_layers, unsigned max_passes,
    unsigned long long max_union_elems, unsigned* changed, int* status) OSH_PUBLIC;
/* No single counterpart in the reference: mesh_adapt (adapt.cpp:82-94) of
   every mesh, unchanged, by nthreads host threads (0 = 4) each issuing on a
   CUDA stream of its own, so that the passes of different meshes overlap on
   the device (one mesh's host read-backs and launch gaps are filled by
   another's kernels). Meshes start largest first while the device-memory
   estimates of the meshes in flight fit budget_bytes (0 = 70% of the free
   device memory; a mesh larger than the budget runs alone). Each mesh ends
   exactly as osh_adapt leaves it, on the stream it had. changed / status as
   for osh_b200_adapt_batch; per-mesh statistics through
   osh_b200_batch_mesh_stats. Meshes need not share dimension or tags. */
int osh_b200_adapt_concurrent(osh_t* meshes, unsigned nmeshes, double size_ratio_floor,
    double good_qual, unsigned nsliver_layers, unsigned max_passes, unsigned nthreads,
    unsigned long long budget_bytes, unsigned* changed, int* status) OSH_PUBLIC;
/* statistics of the last osh_b200_adapt_batch on this thread: unions,
   scheduling steps, passes over whole unions, passes that changed a mesh
   (summed over meshes) and the elements entering those passes */
void osh_b200_batch_stats(unsigned* unions, unsigned* steps, unsigned* union_passes,
    unsigned* mesh_passes, double* elems_in) OSH_PUBLIC;
/* host seconds of the last osh_b200_adapt_batch on this thread (and of the
   serving steps since) spent forming unions, in passes, splitting meshes out */
void osh_b200_batch_times(double* concat, double* passes, double* split) OSH_PUBLIC;
/* per-mesh statistics of the last osh_b200_adapt_batch on this thread, for
   mesh i of that call: passes that changed it and the elements entering them */
void osh_b200_batch_mesh_stats(unsigned i, unsigned* passes, double* elems_in) OSH_PUBLIC;

/* ---- size-field producers ------------------------------------------------ */
/* mesh_element_gradients (element_gradients.cpp:72-91): element field
   "grad_<name>" with 3 components per component of the vertex field name */
void osh_b200_element_gradients(osh_t m, char const* name) OSH_PUBLIC;
/* mesh_recover_by_volume (recover_by_volume.cpp:55-68): vertex field name,
   the volume-weighted average of the element field name around each vertex */
void osh_b200_recover_by_volume(osh_t m, char const* name) OSH_PUBLIC;
/* mesh_size_from_hessian (size_from_hessian.cpp:44-72): vertex field
   "adapt_size" = max(max_h - sum_j weights[j] |H_j|, min_h) from the vertex
   field hess_name (9 components per solution component; weights host array,
   or NULL for all 1) */
void osh_b200_size_from_hessian(osh_t m, char const* hess_name, double const* weights,
    double min_h, double max_h) OSH_PUBLIC;
/* mesh_warp_to_limit (warp_to_limit.cpp:31-81): coordinates += f * warp with
   f = 1, 1/2, 1/4 ... until the minimum element quality is at least
   qual_floor; "warp" keeps the part not yet applied. Returns 1 if the whole
   warp was applied. Where the reference would halve forever (a floor the
   unwarped mesh already fails), this build stops with OSH_B200_E_NOCONVERGE. */
unsigned osh_b200_warp_to_limit(osh_t m, double qual_floor) OSH_PUBLIC;

/* ---- single-precision filter with double recheck ------------------------ */
/* No counterpart in the reference. With the filter on (per mesh, inherited by
   the meshes its passes produce), the edge-length tests of refine_by_size and
   coarsen_by_size and the quality tests of refine_quality, coarsen_quality
   and swap_quality first use a single-precision estimate that carries an
   error bound; a candidate is decided on the estimate only when the bound
   puts it clearly on one side of its threshold, and every value that is kept
   is computed in double. Decisions, and so meshes, equal those without the
   filter. Counters (device-wide): candidates decided on the estimate,
   candidates recomputed in double, the largest |estimate - double| seen and
   how often that exceeded the bound (always 0 when the bound holds). */
void osh_b200_set_fp32_filter(osh_t m, int on) OSH_PUBLIC;
void osh_b200_fp32_stats(unsigned long long* decided, unsigned long long* rechecked,
    double* max_error, unsigned* bound_exceeded) OSH_PUBLIC;
void osh_b200_fp32_stats_reset(void) OSH_PUBLIC;
/* Audit mode (device-wide, off by default; for tests): every decision the
   filter takes on an estimate is also taken in double, and every estimate
   whose double value is computed is checked against its bound. Counters:
   decisions audited, audited decisions the double path takes differently
   (always 0 when the bound holds), estimates checked (bound_exceeded of
   osh_b200_fp32_stats then covers all of them). */
void osh_b200_set_fp32_audit(int on) OSH_PUBLIC;
void osh_b200_fp32_audit_stats(unsigned long long* audited, unsigned long long* flips,
    unsigned long long* checked) OSH_PUBLIC;
/* The filter's device estimates for caller-given inputs, beside the double
   values the passes compute (host arrays). Tets: 12 coordinates each (four
   vertices); est / err: the single-precision quality and its bound (+inf:
   no bound), q64: tet_quality (quality.hpp:68-89). Edges: 6 coordinates and
   2 sizes each; side: +1 / -1 when the estimate places the metric length
   (size.cpp:57-69) above / below thr, 0 undecided; ratio64: the double
   metric length. */
void osh_b200_fp32_probe_tets(unsigned n, double const* host_x, float* host_est,
    float* host_err, double* host_q64) OSH_PUBLIC;
void osh_b200_fp32_probe_edges(unsigned n, double const* host_x, double const* host_h,
    double thr, int* host_side, double* host_ratio64) OSH_PUBLIC;

/* ---- device memory -------------------------------------------------------- */
/* All device memory of this library comes from the current device's default
   memory pool, which keeps what it has grown to. osh_b200_pool_reserve grows
   it to at least `bytes` up front, so that a workload whose meshes grow does
   not pay for growing the pool inside its passes. osh_b200_pool_stats reads
   the bytes the pool holds, the bytes in use and the peak in use (reset to
   the current use when reset_high is nonzero). No counterpart in the
   reference. */
void osh_b200_pool_reserve(unsigned long long bytes) OSH_PUBLIC;
void osh_b200_pool_stats(unsigned long long* reserved, unsigned long long* used,
    unsigned long long* used_high, int reset_high) OSH_PUBLIC;

/* ---- mesh files ------------------------------------------------------------ */
/* write_mesh_vtk_opts (vtk_io.cpp:807-826): ascii != 0 writes ASCII arrays
   (VTK_ASCII); otherwise binary arrays, zlib-compressed when compress != 0
   (the reference's USE_ZLIB build). osh_read_vtk reads all three. */
void osh_b200_write_vtk_opts(osh_t m, char const* filename, int ascii, int compress) OSH_PUBLIC;

/* mesh_has_dim (mesh.cpp:295-298): whether the mesh holds entities of
   dimension dim (vertices always; others once set or derived), without
   deriving them */
unsigned osh_b200_has_dim(osh_t m, unsigned dim) OSH_PUBLIC;

/* order-sensitive 64-bit digest of a mesh (connectivity of every dimension,
   tag names, kinds and data, global numbers), computed on the device; equal
   meshes give equal digests. No counterpart in the reference. */
unsigned long long osh_b200_digest(osh_t m) OSH_PUBLIC;

/* ---- serving: continuous batching of adaptation jobs ------------------- */
/* No counterpart in the reference. A server adapts jobs (a simplex mesh with
   a vertex size field, given in host memory) with mesh_adapt's parameters.
   Jobs wait until the device-memory budget (bytes, estimated from each job's
   size field) admits them; admitted jobs are classified (crease pi/4), join
   the running batch at the next step and leave it when their pass loop ends,
   so jobs that arrive while others run share every launch with them. Each
   result equals what osh_adapt gives the same job alone. Without an engine
   thread (below), call one server from one thread. */
typedef struct osh_b200_server* osh_b200_server_t;
osh_b200_server_t osh_b200_server_new(double size_ratio_floor, double good_qual,
    unsigned nsliver_layers, unsigned max_passes,
    unsigned long long mem_budget_bytes) OSH_PUBLIC;
void osh_b200_server_free(osh_b200_server_t sv) OSH_PUBLIC;
/* queue a job (arrays are copied); returns its id, or -1 */
int osh_b200_server_submit(osh_b200_server_t sv, unsigned dim, unsigned nverts,
    double const* coords, unsigned nelems, unsigned const* conn,
    double const* size) OSH_PUBLIC;
/* largest batch one pass forms, in current elements (default 4e6; 0 = no
   limit): larger batches need fewer launches, smaller ones gather from L2 */
void osh_b200_server_set_union_elems(osh_b200_server_t sv,
    unsigned long long max_elems) OSH_PUBLIC;
/* admit, run one step over every resident job, retire finished jobs;
   returns the number of jobs queued or running, or -1 on error */
int osh_b200_server_step(osh_b200_server_t sv) OSH_PUBLIC;
/* run the steps on an engine thread of the server's own, so that jobs
   submitted from the caller's thread join while others run; after start,
   osh_b200_server_step must not be called. osh_b200_server_wait blocks until
   every submitted job has finished or timeout_s seconds pass (negative: no
   limit) and returns the number of jobs not finished, or -1 on an error (the
   engine stops at its first error; its code and message are then reported
   here). osh_b200_server_stop ends the engine after its current step (also
   done by osh_b200_server_free). Submit, poll, take and the info calls may be
   used from one other thread while the engine runs. */
void osh_b200_server_start(osh_b200_server_t sv) OSH_PUBLIC;
int osh_b200_server_wait(osh_b200_server_t sv, double timeout_s) OSH_PUBLIC;
void osh_b200_server_stop(osh_b200_server_t sv) OSH_PUBLIC;
/* ids of finished jobs not yet reported (at most max_ids); returns the count */
unsigned osh_b200_server_poll(osh_b200_server_t sv, unsigned* ids,
    unsigned max_ids) OSH_PUBLIC;
/* the adapted mesh of a finished job; the caller frees it with osh_free */
osh_t osh_b200_server_take(osh_b200_server_t sv, unsigned id) OSH_PUBLIC;
/* times in seconds since osh_b200_server_new; returns 1 if finished, 0 if
   not yet, -1 for an unknown id */
int osh_b200_server_job_info(osh_b200_server_t sv, unsigned id, double* t_submit,
    double* t_admit, double* t_done, unsigned* passes, double* elems_in,
    int* status) OSH_PUBLIC;
void osh_b200_server_stats(osh_b200_server_t sv, unsigned* steps, unsigned* active,
    unsigned* queued, unsigned long long* reserved_bytes, double* now) OSH_PUBLIC;
/* host seconds spent so far admitting jobs (upload and classification),
   joining them to the running batch, in passes, and retiring finished jobs */
void osh_b200_server_times(osh_b200_server_t sv, double* admit, double* join,
    double* passes, double* retire) OSH_PUBLIC;

/* ---- per-stage selections of one pass, without changing the mesh ------ */
/* Layouts follow refine_by_size / coarsen_common / swap_common: every output
   is a host array sized by the entity counts of the current mesh. */
unsigned osh_b200_refine_sets(osh_t m, double qual_floor,
    unsigned* host_cand, unsigned* host_good, double* host_quals,
    unsigned* host_indset) OSH_PUBLIC;
unsigned osh_b200_coarsen_sets(osh_t m, double qual_floor, double size_floor,
    unsigned* host_codes_size, unsigned* host_codes_class,
    unsigned* host_codes_qual, double* host_quals2, unsigned* host_cand,
    double* host_col_qual, unsigned* host_indset,
    unsigned* host_gen_vert) OSH_PUBLIC;
unsigned osh_b200_swap_sets(osh_t m, double good_qual, unsigned nlayers,
    unsigned* host_slivers, unsigned* host_cand, unsigned* host_interior,
    unsigned* host_good, double* host_quals, unsigned* host_ring_sizes,
    unsigned* host_indset) OSH_PUBLIC;

/* ---- mesh construction -------------------------------------------------- */
/* A reduced-representation mesh (elements only) from host arrays, with a
   "coordinates" vertex field: new_mesh(dim, MESH_REDUCED, 0) +
   mesh_set_ents + mesh_add_tag (mesh.cpp:56-66). */
osh_t osh_b200_new_reduced(unsigned elem_dim, unsigned nverts,
    double const* host_coords, unsigned nelems,
    unsigned const* host_conn) OSH_PUBLIC;
/* mesh_derive_model (derive_model.cpp:444-448) then mesh_set_rep(FULL) */
void osh_b200_derive_model(osh_t m, double crease_angle) OSH_PUBLIC;
/* mesh_make_parallel (mesh.cpp:320-327): single-rank global numbering */
void osh_b200_make_parallel(osh_t m) OSH_PUBLIC;
/* deep copy of a mesh on the same GPU (connectivity, fields, labels, global
   numbers); derived adjacency is rebuilt on demand. No reference
   counterpart: the reference copies meshes only through files. */
osh_t osh_b200_clone(osh_t m) OSH_PUBLIC;

/* n^3 hexahedra of the unit cube, each split into 6 tets like the
   reference's single-cube box (tables.cpp:29-36); interior vertices moved by
   up to pert/n per axis from a splitmix64 stream seeded with `seed`;
   host_center receives the next three draws scaled to [0.3, 0.7]. */
void osh_b200_box(unsigned n, unsigned long seed, double pert,
    double* host_coords, unsigned* host_conn, double* host_center) OSH_PUBLIC;

/* generic tags from host data: type 0 u8, 1 u32, 2 u64, 3 f64 (tag.hpp) */
void osh_b200_add_tag(osh_t m, unsigned dim, char const* name, unsigned type,
    unsigned ncomps, unsigned transfer, void const* host_data) OSH_PUBLIC;
unsigned osh_b200_ntags(osh_t m, unsigned dim) OSH_PUBLIC;
char const* osh_b200_tag_name(osh_t m, unsigned dim, unsigned i) OSH_PUBLIC;
void osh_b200_tag_info(osh_t m, unsigned dim, unsigned i, unsigned* type,
    unsigned* ncomps, unsigned* transfer) OSH_PUBLIC;
void const* osh_b200_tag_data(osh_t m, unsigned dim, unsigned i) OSH_PUBLIC;
void osh_b200_set_globals(osh_t m, unsigned dim,
    unsigned long const* host_globals) OSH_PUBLIC;
/* element dual (mesh_ask_dual, mesh.cpp:252-261), device array */
unsigned const* osh_b200_dual(osh_t m) OSH_PUBLIC;
/* element qualities and edge metric lengths into host arrays */
void osh_b200_qualities(osh_t m, double* host_out) OSH_PUBLIC;
void osh_b200_edge_lengths(osh_t m, double* host_out) OSH_PUBLIC;

/* statistics of the last osh_adapt on this thread: passes that changed the
   mesh and the elements entering them, summed */
void osh_b200_adapt_stats(unsigned* passes, double* elems_in) OSH_PUBLIC;
/* kernels launched by this library so far in the process, and the times it
   waited for the device (stream synchronisations) */
unsigned long long osh_b200_launch_count(void) OSH_PUBLIC;
unsigned long long osh_b200_sync_count(void) OSH_PUBLIC;
/* device allocations made by this library so far, and the host seconds its
   stream synchronisations spent waiting for the device (diagnostics of the
   host side of a pass) */
void osh_b200_host_stats(unsigned long long* allocs, double* sync_wait_seconds) OSH_PUBLIC;
/* self-test of the scans' bounded wait (no counterpart in the reference,
   whose Thrust scan has none): runs one scan whose second tile waits for a
   first tile that never publishes, with a wait limit of spin_limit polls.
   Returns OSH_B200_E_TIMEOUT when the wait gave up and was reported (the
   expected result), 0 if it did not, or another error code; the device
   stays usable afterwards. */
int osh_b200_selftest_scan_wait(unsigned spin_limit) OSH_PUBLIC;
/* the passes' exclusive scan over device arrays (replaces uints_exscan,
   ints.cpp:45-59, a Thrust scan there): out[0..n] with out[0] = 0 and
   out[n] the total of in[0..n), 32-bit wrap-around sums, queued on `stream`
   (a cudaStream_t; 0 is the legacy default stream). With check != 0 the
   call waits for the stream and returns OSH_B200_E_TIMEOUT if a bounded
   look-back wait gave up; with check == 0 it returns once the scan is
   queued. in and out may not overlap. Returns 0 or an error code. */
int osh_b200_exscan_u32(unsigned const* in, unsigned* out, unsigned n, void* stream,
    int check) OSH_PUBLIC;
/* run all further work of mesh m on the CUDA stream `stream` (a
   cudaStream_t; 0 is the legacy default stream); the caller keeps it alive */
void osh_b200_set_stream(osh_t m, void* stream) OSH_PUBLIC;
/* before the caller destroys a stream it gave to osh_b200_set_stream: frees
   the scratch the library keeps for that stream (in the stream's order), so
   that it does not outlive it. No mesh may use the stream afterwards. */
void osh_b200_release_stream(void* stream) OSH_PUBLIC;

/* ---- launch shapes (tuning table) ------------------------------------------ */
/* No counterpart in the reference (its loops launch 256 threads per block,
   loop_cuda.hpp:28-53). Lanes per row of the long-row kernels, threads per
   block and scan tile sizes come from a table: defaults, overridden once at
   load by the file named by OSH_B200_TUNING or else tuning.txt beside the
   library ("name value" lines, written by omega_h_v1_b200/tune.py, which
   times each candidate with CUDA events on the GPU it runs on). Every allowed
   value gives the same meshes. get/set/load return 0 or OSH_B200_E_ARG
   (unknown name, a value the key does not allow, or a bad line in the file:
   then nothing of the file is applied) / OSH_B200_E_IO (unreadable file). */
unsigned osh_b200_tuning_count(void) OSH_PUBLIC;
char const* osh_b200_tuning_name(unsigned i) OSH_PUBLIC;
int osh_b200_tuning_get(char const* name, unsigned* value) OSH_PUBLIC;
int osh_b200_tuning_set(char const* name, unsigned value) OSH_PUBLIC;
int osh_b200_tuning_load(char const* path) OSH_PUBLIC;

/* ---- per-kernel event probes (bench instrumentation) -------------------- */
/* Bit i of mask enables probe i: each launch of that kernel is bracketed by
   CUDA events on its stream and credited with its algorithmic bytes. */
void osh_b200_probe_enable(unsigned mask) OSH_PUBLIC;
void osh_b200_probe_reset(void) OSH_PUBLIC;
unsigned osh_b200_probe_count(void) OSH_PUBLIC;
char const* osh_b200_probe_name(unsigned id) OSH_PUBLIC;
void osh_b200_probe_read(unsigned id, unsigned* launches, double* total_ms,
    double* total_bytes) OSH_PUBLIC;

/* ---- upward adjacency without device allocation -------------------------- */
/* No counterpart in the reference. For callers that cannot allocate device
   memory when they need the adjacency: host callbacks and real-time loops
   that must not wait on the allocator, and host codes that give the GPU a
   fixed memory budget and own every byte of it.
   Computes the same upward adjacency as osh_up_offs / osh_up / osh_up_dirs
   (rows sorted by use index) from a device array lows_of_highs of
   nuses = nhighs * deg(high_dim, low_dim) entries into caller-allocated
   device arrays offsets[nlows + 1], highs_of_lows[nuses] and
   directions[nuses], enqueued on `stream` (a cudaStream_t, 0 = legacy
   default stream) without synchronising. It calls no allocator: its scratch
   is one fixed device array inside the library (about 8.4 MB, held by every
   GPU that loads the library until the process exits), so the sizes are
   capped at OSH_B200_NOALLOC_MAX_USES uses and OSH_B200_NOALLOC_MAX_LOWS
   rows; larger requests return OSH_B200_E_ARG without launching anything.
   The first call on each device looks up the array's device address (with
   that device current), so make it before any stream capture on that
   device. Every call shares the one array and clears what it needs; calls
   that may run at the same time on the GPU (different streams, no ordering
   between them) race and must not be issued. Failures found on the device
   (an entry of lows_of_highs not below nlows, a bounded wait that gave up)
   write nothing through a computed index and leave 0xffffffff in
   offsets[nlows], which holds nuses after a successful call: read it once
   the stream's work is done. Returns 0, or the error code also recorded
   for osh_b200_last_error(). */
#define OSH_B200_NOALLOC_MAX_USES (1u << 20)
#define OSH_B200_NOALLOC_MAX_LOWS (1u << 20)
int osh_b200_up_from_down_noalloc(unsigned high_dim, unsigned low_dim,
    unsigned nhighs, unsigned nlows, unsigned const* lows_of_highs,
    unsigned* offsets, unsigned* highs_of_lows, unsigned* directions,
    void* stream) OSH_PUBLIC;

/* ---- memory helpers ----------------------------------------------------- */
/* The arrays osh_build_ents, osh_new_field and osh_new_label return are
   device memory, ready for these copies when the call returns. */
void osh_b200_copy_to_host(void* host_dst, void const* dev_src, size_t bytes) OSH_PUBLIC;
void osh_b200_copy_to_device(void* dev_dst, void const* host_src, size_t bytes) OSH_PUBLIC;
/* The same copies queued on mesh m's stream (no counterpart in the
   reference): they return at once, run in order with m's work, and the host
   buffer must stay valid, and unchanged for an upload, until the stream has
   passed the copy (osh_b200_synchronize(m), or any call that returns
   results). Page-locked host memory makes them asynchronous. */
void osh_b200_copy_to_host_async(osh_t m, void* host_dst, void const* dev_src, size_t bytes)
    OSH_PUBLIC;
void osh_b200_copy_to_device_async(osh_t m, void* dev_dst, void const* host_src, size_t bytes)
    OSH_PUBLIC;
void osh_b200_synchronize(osh_t m) OSH_PUBLIC;

/* polygon triangulation table used by edge swapping (edge_swap.cpp:21-228):
   per ring size 3..7, the triangles (3 ring-vertex ids each) of every
   triangulation and its interior edges. Returns 0 for other sizes. */
unsigned osh_b200_swap_table(unsigned ring_size, unsigned* ntri,
    unsigned* nmesh, unsigned* nint, unsigned* host_tris,
    unsigned* host_iedges) OSH_PUBLIC;

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif
