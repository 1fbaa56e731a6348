/*
 * omega_h.h -- C ABI of the B200 mesh-adaptation library (libosh_b200.so).
 *
 * Drop-in for Omega_h v1's public C API (reference: include/omega_h.h:1-84,
 * implemented in omega_h.cpp). Same names, argument meaning and return
 * values. As with the reference's CUDA build, every array returned or
 * accepted here lives in device memory of the current GPU; use
 * osh_b200_copy_to_host / osh_b200_copy_to_device (omega_h_b200.h) or
 * cudaMemcpy to move data. Arrays returned by the API belong to the mesh and
 * become invalid after any call that modifies the mesh.
 *
 * Errors: the reference asserts or aborts; this library never aborts. A
 * failed call leaves the mesh unchanged where it can, returns 0 / NULL, and
 * records a code readable with osh_b200_last_error().
 */
#ifndef OMEGA_H_H
#define OMEGA_H_H

#define OSH_PUBLIC __attribute__((visibility("default")))

#ifdef __cplusplus
extern "C" {
#endif

typedef struct osh_mesh* osh_t;

/* omega_h.h:12-13 -- no MPI here; both only check the CUDA runtime. */
void osh_init(int* argc, char*** argv) OSH_PUBLIC;
void osh_fini(void) OSH_PUBLIC;

/* omega_h.h:15 */
void osh_free(osh_t m) OSH_PUBLIC;

/* omega_h.h:17-18 (omega_h.cpp:127-154, vtk_io.cpp:787-830) -- the
   reference's VTU format byte for byte. "x.vtu" is a serial mesh; "x.pvtu"
   names the parallel index file of the single piece "x.vtu" (one rank).
   osh_write_vtk writes binary (base64) arrays without compression, as the
   reference's default build does; osh_b200_write_vtk_opts (omega_h_b200.h)
   selects ASCII or zlib. A missing or malformed file sets OSH_B200_E_IO. */
osh_t osh_read_vtk(char const* filename) OSH_PUBLIC;
void osh_write_vtk(osh_t m, char const* filename) OSH_PUBLIC;

/* omega_h.h:20-21 -- an empty full-topology, single-rank parallel mesh
   (omega_h.cpp:177-182); osh_build_ents returns device memory to fill. */
osh_t osh_new(unsigned elem_dim) OSH_PUBLIC;
unsigned* osh_build_ents(osh_t m, unsigned ent_dim, unsigned nents) OSH_PUBLIC;

/* omega_h.h:23-26 */
unsigned osh_dim(osh_t m) OSH_PUBLIC;
unsigned osh_nelems(osh_t m) OSH_PUBLIC;
unsigned osh_nverts(osh_t m) OSH_PUBLIC;
unsigned osh_count(osh_t m, unsigned dim) OSH_PUBLIC;

/* omega_h.h:28-33 -- adjacency, derived on first request */
unsigned const* osh_down(osh_t m, unsigned high_dim, unsigned low_dim) OSH_PUBLIC;
unsigned const* osh_up(osh_t m, unsigned low_dim, unsigned high_dim) OSH_PUBLIC;
unsigned const* osh_up_offs(osh_t m, unsigned low_dim, unsigned high_dim) OSH_PUBLIC;
unsigned const* osh_up_dirs(osh_t m, unsigned low_dim, unsigned high_dim) OSH_PUBLIC;
unsigned const* osh_star(osh_t m, unsigned low_dim, unsigned high_dim) OSH_PUBLIC;
unsigned const* osh_star_offs(osh_t m, unsigned low_dim, unsigned high_dim) OSH_PUBLIC;

/* omega_h.h:35 */
double const* osh_coords(osh_t m) OSH_PUBLIC;

/* omega_h.h:37-39 -- single rank: every entity is owned by rank 0 */
unsigned const* osh_own_rank(osh_t m, unsigned dim) OSH_PUBLIC;
unsigned const* osh_own_id(osh_t m, unsigned dim) OSH_PUBLIC;
unsigned long const* osh_global(osh_t m, unsigned dim) OSH_PUBLIC;

/* omega_h.h:41-46 */
enum osh_transfer {
  OSH_TRANSFER_NOT,
  OSH_TRANSFER_POINTWISE,
  OSH_TRANSFER_CONSERVE,
  OSH_TRANSFER_INHERIT
};

/* omega_h.h:48-55 */
double* osh_new_field(osh_t m, unsigned dim, char const* name,
    unsigned ncomps, enum osh_transfer tt) OSH_PUBLIC;
double* osh_get_field(osh_t m, unsigned dim, char const* name) OSH_PUBLIC;
void osh_free_field(osh_t m, unsigned dim, char const* name) OSH_PUBLIC;

unsigned osh_nfields(osh_t om, unsigned dim) OSH_PUBLIC;
char const* osh_field(osh_t m, unsigned dim, unsigned i) OSH_PUBLIC;
unsigned osh_components(osh_t m, unsigned dim, char const* name) OSH_PUBLIC;

/* omega_h.h:57-59 */
unsigned* osh_new_label(osh_t m, unsigned dim, char const* name, unsigned ncomps) OSH_PUBLIC;
unsigned* osh_get_label(osh_t m, unsigned dim, char const* name) OSH_PUBLIC;
void osh_free_label(osh_t m, unsigned dim, char const* name) OSH_PUBLIC;

/* omega_h.h:61 */
unsigned long* osh_new_global(osh_t m, unsigned dim) OSH_PUBLIC;

/* omega_h.h:63-64 -- exchanges with other ranks; a no-op on one rank */
void osh_accumulate_to_owner(osh_t m, unsigned dim, char const* name) OSH_PUBLIC;
void osh_conform(osh_t m, unsigned dim, char const* name) OSH_PUBLIC;

/* omega_h.h:66-67 -- `marked` is a device array of osh_count(m, ent_dim) */
void osh_mark_classified(osh_t m, unsigned ent_dim,
    unsigned class_dim, unsigned class_id, unsigned* marked) OSH_PUBLIC;

/* omega_h.h:69-70 -- one rank has nothing to ghost; the count is recorded */
void osh_ghost(osh_t m, unsigned nlayers) OSH_PUBLIC;
unsigned osh_num_ghost_layers(osh_t m) OSH_PUBLIC;

/* omega_h.h:72-76 (omega_h.cpp:1005-1016): refine, coarsen and fix slivers;
   returns 0 when the connectivity did not change. Needs the "coordinates"
   and "adapt_size" vertex fields and class_dim / class_id labels. */
unsigned osh_adapt(osh_t m,
    double size_ratio_floor,
    double good_element_quality,
    unsigned nsliver_layers,
    unsigned max_passes) OSH_PUBLIC;

/* omega_h.h:78 -- per-vertex longest adjacent edge as a size field */
void osh_identity_size(osh_t m, char const* name) OSH_PUBLIC;

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif
