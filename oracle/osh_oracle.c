/*
 * osh_oracle.c -- TEST INFRASTRUCTURE ONLY. This file is the checker for the
 * CUDA adaptation pass; it is never linked into, loaded by, or timed as the
 * product. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg use it (through oracle/oracle.py).
 *
 * A plain-C, serial restatement of Omega_h v1's mesh-adaptation pass
 * (refine_by_size / coarsen_by_size / coarsen_slivers / swap_slivers /
 * mesh_adapt) and of everything those passes call: the lazy adjacency cache,
 * upward / downward / star / dual derivation, classification, qualities,
 * Luby independent sets, the topology rebuilds and the field transfers.
 * Each function cites the reference file:line it follows. Floating-point
 * expressions keep the reference's operation order so that results are
 * bit-identical to the reference built with -O2 on x86-64 (no FMA; this file
 * is compiled with -ffp-contract=off).
 *
 * Where the reference's serial and OpenMP builds differ (the serial
 * doubles_min skips element 0, doubles.cpp:111-118), this restatement follows
 * the OpenMP/CUDA semantics: the minimum over all elements.
 *
 * Parity pin: tests/test_oracle.py runs this restatement and the
 * reference itself (compiled from its own sources into oracle/_ref/ by
 * oracle/Makefile) on the same seeded inputs and requires identical meshes.
 */
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "osh_oracle_tables.h"

#define INV 0xffffffffu
#define MAX_ITERATIONS 100 /* indset.cpp:33 */
#define MAX_EDGE_SWAP 7    /* edge_swap.hpp:6 */
#define MAX_PTS 16         /* qr.hpp:6 */
#define MAX_NCOMPS 32      /* coarsen_conserve.cpp:10 */
#define ORACLE_PI 3.14159265359 /* algebra.hpp:8 */

typedef unsigned u32;
typedef unsigned long u64;

enum { T_U8, T_U32, T_U64, T_F64 };                 /* tag.hpp:9-14 */
enum { X_NOT, X_POINTWISE, X_CONSERVE, X_INHERIT }; /* omega_h.h:41-46 */
enum { DONT_COLLAPSE = 0, COLLAPSE_BOTH = 3 };      /* collapse_codes.hpp:9-14 */
enum { NOT_IN_SET = 0, IN_SET = 1, UNKNOWN = 2 };   /* indset.cpp:35-39 */
enum { E_OK = 0, E_NOCONVERGE = 1, E_MAXOPS = 2, E_BAD = 3 };

/* ------------------------------------------------------------------------ */
/* topology tables (tables.cpp:77-193)                                       */

static const u32 DEG[4][4] = {
  {1, 0, 0, 0}, {2, 1, 0, 0}, {3, 3, 1, 0}, {4, 6, 4, 1}};
static const u32 TRI_EV[3][2] = {{0, 1}, {1, 2}, {2, 0}};
static const u32 TET_EV[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
static const u32 TET_FV[4][3] = {{0, 1, 2}, {1, 0, 3}, {2, 1, 3}, {0, 2, 3}};
static const u32 TET_FE[4][3] = {{0, 1, 2}, {0, 3, 4}, {1, 4, 5}, {2, 5, 3}};
static const u32 OPP_EV[2] = {1, 0};
static const u32 OPP_FV[3] = {1, 2, 0};
static const u32 OPP_FE[3] = {2, 0, 1};
static const u32 OPP_RV[4] = {2, 3, 1, 0};
static const u32 OPP_RE[6] = {5, 3, 4, 1, 2, 0};
static const u32 OPP_RF[4] = {3, 2, 0, 1};

/* the_canonical_orders[elem][ent][sub][j][k]: local index (in the element)
   of the k-th sub-entity (of dimension sub) of the element's j-th entity of
   dimension ent. */
static u32 co(u32 elem, u32 ent, u32 sub, u32 j, u32 k)
{
  if (ent == elem)
    return k;
  if (sub == ent)
    return j;
  if (ent == 1 && sub == 0)
    return (elem == 2) ? TRI_EV[j][k] : TET_EV[j][k];
  if (ent == 2 && sub == 0)
    return TET_FV[j][k];
  return TET_FE[j][k]; /* elem 3, ent 2, sub 1 */
}

/* the_opposite_orders[elem][dim][j] */
static u32 opp(u32 elem, u32 dim, u32 j)
{
  switch (elem) {
    case 1: return OPP_EV[j];
    case 2: return dim == 0 ? OPP_FV[j] : OPP_FE[j];
    default:
      if (dim == 0) return OPP_RV[j];
      if (dim == 1) return OPP_RE[j];
      return OPP_RF[j];
  }
}

/* single-cube split into 6 tets around diagonal 0-6 (tables.cpp:29-36) */
static const u32 CUBE_SPLIT[6][4] = {
  {0, 1, 2, 6}, {2, 3, 0, 6}, {0, 3, 7, 6},
  {7, 4, 0, 6}, {0, 4, 5, 6}, {5, 1, 0, 6}};
static const u32 CUBE_CORNER[8][3] = {
  {0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
  {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

/* ------------------------------------------------------------------------ */
/* memory and array helpers (arrays.cpp, ints.cpp)                           */

static void* xmalloc(size_t n)
{
  void* p = malloc(n ? n : 1);
  if (!p) {
    fprintf(stderr, "oracle: out of memory\n");
    abort();
  }
  return p;
}
#define NEW(T, n) ((T*)xmalloc(sizeof(T) * (size_t)(n)))

static u32* u32_filled(u32 n, u32 v)
{
  u32* a = NEW(u32, n);
  for (u32 i = 0; i < n; ++i) a[i] = v;
  return a;
}

static u32* u32_copy(u32 const* a, u32 n)
{
  u32* b = NEW(u32, n);
  memcpy(b, a, sizeof(u32) * n);
  return b;
}

/* uints_exscan: n+1 outputs, total at [n] (ints.cpp:22-33) */
static u32* u32_exscan(u32 const* a, u32 n)
{
  u32* o = NEW(u32, n + 1);
  u32 s = 0;
  o[0] = 0;
  for (u32 i = 0; i < n; ++i) {
    s += a[i];
    o[i + 1] = s;
  }
  return o;
}

static u32 u32_max(u32 const* a, u32 n)
{
  u32 m = 0;
  for (u32 i = 0; i < n; ++i)
    if (a[i] > m) m = a[i];
  return m;
}

/* uints_negate_offsets (ints.cpp:227-235) */
static u32* negate_offsets(u32 const* offs, u32 n)
{
  u32* t = NEW(u32, n);
  for (u32 i = 0; i < n; ++i) t[i] = !(offs[i + 1] - offs[i]);
  u32* o = u32_exscan(t, n);
  free(t);
  return o;
}

/* expand_array (arrays.cpp:170-192), element size esz bytes */
static void* expand_bytes(void const* a, u32 const* offs, u32 n, u32 width,
    size_t esz)
{
  char* out = (char*)xmalloc((size_t)offs[n] * width * esz);
  char const* in = (char const*)a;
  size_t row = (size_t)width * esz;
  for (u32 i = 0; i < n; ++i)
    for (u32 j = offs[i]; j < offs[i + 1]; ++j)
      memcpy(out + (size_t)j * row, in + (size_t)i * row, row);
  return out;
}

static size_t tag_esz(u32 type)
{
  switch (type) {
    case T_U8: return 1;
    case T_U32: return 4;
    case T_U64: return 8;
    default: return 8;
  }
}

/* ------------------------------------------------------------------------ */
/* tags (tag.cpp:34-118)                                                     */

typedef struct {
  char* name;
  u32 type, ncomps, transfer;
  void* data;
} otag;

typedef struct {
  u32 n, cap;
  otag** at;
} otags;

static otag* tags_find(otags* ts, char const* name)
{
  for (u32 i = 0; i < ts->n; ++i)
    if (!strcmp(ts->at[i]->name, name)) return ts->at[i];
  return 0;
}

static otag* tags_add(otags* ts, u32 type, char const* name, u32 ncomps,
    u32 transfer, void* data)
{
  if (tags_find(ts, name)) {
    fprintf(stderr, "oracle: duplicate tag %s\n", name);
    abort();
  }
  otag* t = NEW(otag, 1);
  t->name = NEW(char, strlen(name) + 1);
  strcpy(t->name, name);
  t->type = type;
  t->ncomps = ncomps;
  t->transfer = transfer;
  t->data = data;
  if (ts->n == ts->cap) {
    ts->cap = ts->cap ? ts->cap * 2 : 8;
    ts->at = (otag**)realloc(ts->at, sizeof(otag*) * ts->cap);
  }
  ts->at[ts->n++] = t;
  return t;
}

static void tag_free(otag* t)
{
  free(t->name);
  free(t->data);
  free(t);
}

static void tags_remove(otags* ts, char const* name)
{
  for (u32 i = 0; i < ts->n; ++i)
    if (!strcmp(ts->at[i]->name, name)) {
      tag_free(ts->at[i]);
      for (; i + 1 < ts->n; ++i) ts->at[i] = ts->at[i + 1];
      ts->n--;
      return;
    }
}

static void tags_clear(otags* ts)
{
  for (u32 i = 0; i < ts->n; ++i) tag_free(ts->at[i]);
  free(ts->at);
  ts->at = 0;
  ts->n = ts->cap = 0;
}

/* ------------------------------------------------------------------------ */
/* mesh store with lazy adjacency cache (mesh.cpp:27-334)                    */

typedef struct {
  u32* offs;
  u32* adj;
  u32* dirs;
} oup;

typedef struct {
  u32* offs;
  u32* adj;
} ograph;

typedef struct omesh {
  u32 dim;
  int full;
  int parallel;
  u32 counts[4];
  u32* down[4][4];
  oup* up[4][4];
  ograph* star[4][4];
  u32* dual;
  otags tags[4];
  u64* globals[4];
  int err;
} omesh;

static omesh* mesh_new(u32 dim, int full, int parallel)
{
  omesh* m = NEW(omesh, 1);
  memset(m, 0, sizeof(*m));
  m->dim = dim;
  m->full = full;
  m->parallel = parallel;
  return m;
}

static void mesh_clear(omesh* m)
{
  for (u32 h = 0; h < 4; ++h)
    for (u32 l = 0; l < 4; ++l) {
      free(m->down[h][l]);
      if (m->up[l][h]) {
        free(m->up[l][h]->offs);
        free(m->up[l][h]->adj);
        free(m->up[l][h]->dirs);
        free(m->up[l][h]);
      }
      if (m->star[l][h]) {
        free(m->star[l][h]->offs);
        free(m->star[l][h]->adj);
        free(m->star[l][h]);
      }
    }
  free(m->dual);
  for (u32 d = 0; d < 4; ++d) {
    tags_clear(&m->tags[d]);
    free(m->globals[d]);
  }
}

/* overwrite_mesh (mesh.cpp:329-334) */
static void mesh_overwrite(omesh* m, omesh* with)
{
  int err = m->err;
  mesh_clear(m);
  *m = *with;
  m->err = err;
  free(with);
}

static void set_ents(omesh* m, u32 dim, u32 n, u32* verts)
{
  m->counts[dim] = n;
  m->down[dim][0] = verts;
}

static int has_dim(omesh* m, u32 dim)
{
  return dim == 0 || m->down[dim][0] != 0;
}

static u32 const* ask_down(omesh* m, u32 high, u32 low);
static oup* ask_up(omesh* m, u32 low, u32 high);
static ograph* ask_star(omesh* m, u32 low, u32 high);
static u32 const* ask_dual(omesh* m);

static u32 count(omesh* m, u32 dim)
{
  if (dim > m->dim) return 0;
  if (dim) ask_down(m, dim, 0);
  return m->counts[dim];
}

static double const* coords_of(omesh* m)
{
  return (double const*)tags_find(&m->tags[0], "coordinates")->data;
}

/* invert_map, CPU flavour (invert_map.cpp:118-136): each row ends up sorted
   by use index, which a stable counting sort produces directly. */
static void invert_map(u32 nin, u32 const* in, u32 nout, u32** p_out,
    u32** p_offs)
{
  u32* cnt = u32_filled(nout, 0);
  for (u32 i = 0; i < nin; ++i) cnt[in[i]]++;
  u32* offs = u32_exscan(cnt, nout);
  for (u32 i = 0; i < nout; ++i) cnt[i] = 0;
  u32* out = NEW(u32, nin);
  for (u32 i = 0; i < nin; ++i) {
    u32 d = in[i];
    out[offs[d] + cnt[d]++] = i;
  }
  free(cnt);
  *p_out = out;
  *p_offs = offs;
}

/* up_from_down (up_from_down.cpp:24-47) */
static oup* up_from_down(u32 high, u32 low, u32 nhighs, u32 nlows,
    u32 const* lows_of_highs)
{
  u32 lph = DEG[high][low];
  u32 nuses = nhighs * lph;
  oup* u = NEW(oup, 1);
  invert_map(nuses, lows_of_highs, nlows, &u->adj, &u->offs);
  u->dirs = NEW(u32, nuses);
  for (u32 i = 0; i < nuses; ++i) {
    u32 both = u->adj[i];
    u->adj[i] = both / lph;
    u->dirs[i] = both % lph;
  }
  return u;
}

/* find_edge_up / find_tri_up (find_by_verts.hpp:14-55) */
static u32 find_by_verts(u32 low, u32 const* w, u32 const* verts_of_lows,
    oup const* lows_of_verts)
{
  u32 v0 = w[0];
  if (low == 1) {
    for (u32 i = lows_of_verts->offs[v0]; i < lows_of_verts->offs[v0 + 1]; ++i) {
      u32 e = lows_of_verts->adj[i];
      u32 d = lows_of_verts->dirs[i];
      if (verts_of_lows[e * 2 + (1 - d)] == w[1]) return e;
    }
  } else {
    for (u32 i = lows_of_verts->offs[v0]; i < lows_of_verts->offs[v0 + 1]; ++i) {
      u32 t = lows_of_verts->adj[i];
      u32 d = lows_of_verts->dirs[i];
      u32 const* tv = verts_of_lows + t * 3;
      u32 a = tv[(d + 1) % 3], b = tv[(d + 2) % 3];
      if ((a == w[1] && b == w[2]) || (a == w[2] && b == w[1])) return t;
    }
  }
  return INV;
}

/* mesh_reflect_down / reflect_down_entity (reflect_down.cpp:13-81) */
static u32* reflect_down(omesh* m, u32 high, u32 low)
{
  u32 nh = count(m, high);
  u32 const* voh = ask_down(m, high, 0);
  oup* lov = ask_up(m, 0, low);
  u32 const* vol = ask_down(m, low, 0);
  u32 vph = DEG[high][0], lph = DEG[high][low], vpl = DEG[low][0];
  u32* out = NEW(u32, nh * lph);
  for (u32 i = 0; i < nh; ++i)
    for (u32 j = 0; j < lph; ++j) {
      u32 w[3];
      for (u32 k = 0; k < vpl; ++k) w[k] = voh[i * vph + co(high, low, 0, j, k)];
      out[i * lph + j] = find_by_verts(low, w, vol, lov);
    }
  return out;
}

/* bridge_graph_general (bridge_graph.cpp:47-80) */
static void bridge_graph(u32 n, u32 const* offs, u32 const* adj, u32* p_nedges,
    u32** p_verts_of_edges, u32** p_dirs)
{
  u32* deg = NEW(u32, n);
  for (u32 i = 0; i < n; ++i) {
    u32 d = 0;
    for (u32 j = offs[i]; j < offs[i + 1]; ++j)
      if (i < adj[j]) ++d;
    deg[i] = d;
  }
  u32* bo = u32_exscan(deg, n);
  free(deg);
  u32 ne = bo[n];
  u32* voe = NEW(u32, ne * 2);
  u32* dirs = p_dirs ? NEW(u32, ne) : 0;
  for (u32 i = 0; i < n; ++i) {
    u32 e = bo[i];
    for (u32 j = offs[i]; j < offs[i + 1]; ++j)
      if (i < adj[j]) {
        voe[e * 2 + 0] = i;
        voe[e * 2 + 1] = adj[j];
        if (dirs) dirs[e] = j - offs[i];
        ++e;
      }
  }
  free(bo);
  *p_nedges = ne;
  *p_verts_of_edges = voe;
  if (p_dirs) *p_dirs = dirs;
}

/* mesh_ask_down (mesh.cpp:136-181) */
static u32 const* ask_down(omesh* m, u32 high, u32 low)
{
  if (m->down[high][low]) return m->down[high][low];
  if (low == high) {
    u32 n = m->counts[high];
    u32* a = NEW(u32, n);
    for (u32 i = 0; i < n; ++i) a[i] = i;
    m->down[high][low] = a;
  } else if (low > 0) {
    m->down[high][low] = reflect_down(m, high, low);
  } else if (high == 1 && m->dim == 3) {
    /* edges in 3D from the vertex star (mesh.cpp:160-168) */
    ograph* vv = ask_star(m, 0, m->dim);
    u32 ne, *voe;
    bridge_graph(m->counts[0], vv->offs, vv->adj, &ne, &voe, 0);
    set_ents(m, 1, ne, voe);
  } else {
    /* sides from the element dual (mesh.cpp:169-179, derive_sides.cpp) */
    u32 const* dual = ask_dual(m);
    u32 ne = m->counts[m->dim];
    u32 spe = DEG[m->dim][m->dim - 1];
    u32* offs = NEW(u32, ne + 1);
    for (u32 i = 0; i <= ne; ++i) offs[i] = i * spe;
    u32 ns, *eos, *esos;
    bridge_graph(ne, offs, dual, &ns, &eos, &esos);
    free(offs);
    u32 const* voe = m->down[m->dim][0];
    u32 vpe = DEG[m->dim][0], vps = DEG[m->dim - 1][0];
    u32* vos = NEW(u32, ns * vps);
    for (u32 s = 0; s < ns; ++s) {
      u32 e = eos[s * 2];
      for (u32 j = 0; j < vps; ++j)
        vos[s * vps + j] = voe[e * vpe + co(m->dim, m->dim - 1, 0, esos[s], j)];
    }
    free(eos);
    free(esos);
    set_ents(m, m->dim - 1, ns, vos);
  }
  return m->down[high][low];
}

/* mesh_ask_up (mesh.cpp:190-217) */
static oup* ask_up(omesh* m, u32 low, u32 high)
{
  if (m->up[low][high]) return m->up[low][high];
  if (low == high) {
    u32 n = m->counts[high];
    oup* u = NEW(oup, 1);
    u->offs = NEW(u32, n + 1);
    for (u32 i = 0; i <= n; ++i) u->offs[i] = i;
    u->adj = u32_copy(u->offs, n);
    u->dirs = u32_filled(n, 0);
    m->up[low][high] = u;
  } else {
    u32 const* loh = ask_down(m, high, low);
    m->up[low][high] = up_from_down(high, low, m->counts[high],
        m->counts[low], loh);
  }
  return m->up[low][high];
}

static int has_u32(u32 const* a, u32 n, u32 e)
{
  for (u32 i = 0; i < n; ++i)
    if (a[i] == e) return 1;
  return 0;
}

/* star graphs (star.cpp:14-315) */
static ograph* get_star(omesh* m, u32 low, u32 high)
{
  ograph* g = NEW(ograph, 1);
  if (low == 0 && high == m->dim && m->dim != 1 && has_dim(m, 1)) {
    free(g);
    return get_star(m, 0, 1);
  }
  if (low == 0 && high == 1) {
    /* get_vertex_edge_star (star.cpp:135-160) */
    u32 nv = count(m, 0);
    u32 const* voe = ask_down(m, 1, 0);
    oup* eov = ask_up(m, 0, 1);
    g->offs = u32_copy(eov->offs, nv + 1);
    g->adj = NEW(u32, eov->offs[nv]);
    for (u32 j = 0; j < eov->offs[nv]; ++j)
      g->adj[j] = voe[eov->adj[j] * 2 + (1 - eov->dirs[j])];
    return g;
  }
  if (low == 1 && high == 2) {
    /* get_edge_triangle_star (star.cpp:189-218) */
    u32 ne = count(m, 1);
    u32 const* eot = ask_down(m, 2, 1);
    oup* toe = ask_up(m, 1, 2);
    g->offs = NEW(u32, ne + 1);
    for (u32 i = 0; i <= ne; ++i) g->offs[i] = toe->offs[i] * 2;
    g->adj = NEW(u32, toe->offs[ne] * 2);
    for (u32 j = 0; j < toe->offs[ne]; ++j) {
      u32 t = toe->adj[j], d = toe->dirs[j];
      g->adj[j * 2 + 0] = eot[t * 3 + (d + 1) % 3];
      g->adj[j * 2 + 1] = eot[t * 3 + (d + 2) % 3];
    }
    return g;
  }
  if (low == 1 && high == 3 && has_dim(m, 2)) {
    /* get_edge_tet_star (star.cpp:255-293) */
    ograph* ts = get_star(m, 1, 2);
    u32 ne = count(m, 1);
    u32 const* eor = ask_down(m, 3, 1);
    oup* roe = ask_up(m, 1, 3);
    u32* deg = NEW(u32, ne);
    for (u32 i = 0; i < ne; ++i)
      deg[i] = (ts->offs[i + 1] - ts->offs[i]) + (roe->offs[i + 1] - roe->offs[i]);
    g->offs = u32_exscan(deg, ne);
    free(deg);
    g->adj = NEW(u32, g->offs[ne]);
    for (u32 i = 0; i < ne; ++i) {
      u32 o = g->offs[i];
      for (u32 j = ts->offs[i]; j < ts->offs[i + 1]; ++j) g->adj[o++] = ts->adj[j];
      for (u32 j = roe->offs[i]; j < roe->offs[i + 1]; ++j)
        g->adj[o++] = eor[roe->adj[j] * 6 + OPP_RE[roe->dirs[j]]];
    }
    free(ts->offs);
    free(ts->adj);
    free(ts);
    return g;
  }
  /* get_star_general (star.cpp:14-111) */
  u32 nl = count(m, low);
  oup* hol = ask_up(m, low, high);
  u32 const* loh = ask_down(m, high, low);
  u32 lph = DEG[high][low];
  u32* deg = NEW(u32, nl);
  u32 cap = 64;
  u32* buf = NEW(u32, cap);
  for (int pass = 0; pass < 2; ++pass) {
    for (u32 i = 0; i < nl; ++i) {
      u32 rowcap = (hol->offs[i + 1] - hol->offs[i]) * lph;
      if (rowcap > cap) {
        cap = rowcap;
        buf = (u32*)realloc(buf, sizeof(u32) * cap);
      }
      u32 size = 0;
      for (u32 j = hol->offs[i]; j < hol->offs[i + 1]; ++j) {
        u32 h = hol->adj[j];
        for (u32 k = 0; k < lph; ++k) {
          u32 s = loh[h * lph + k];
          if (s == i) continue;
          if (!has_u32(buf, size, s)) buf[size++] = s;
        }
      }
      if (pass == 0)
        deg[i] = size;
      else
        memcpy(g->adj + g->offs[i], buf, sizeof(u32) * size);
    }
    if (pass == 0) {
      g->offs = u32_exscan(deg, nl);
      g->adj = NEW(u32, g->offs[nl]);
    }
  }
  free(buf);
  free(deg);
  return g;
}

/* mesh_ask_star (mesh.cpp:226-244) */
static ograph* ask_star(omesh* m, u32 low, u32 high)
{
  if (m->star[low][high]) return m->star[low][high];
  if (low == high) {
    ograph* g = NEW(ograph, 1);
    g->offs = u32_filled(m->counts[low] + 1, 0);
    g->adj = 0;
    m->star[low][high] = g;
  } else {
    m->star[low][high] = get_star(m, low, high);
  }
  return m->star[low][high];
}

/* dual_from_sides / dual_from_verts (dual.cpp:36-168) */
static u32 const* ask_dual(omesh* m)
{
  if (m->dual) return m->dual;
  u32 dim = m->dim, ne = count(m, dim), spe = DEG[dim][dim - 1];
  u32* out = NEW(u32, ne * spe);
  if (has_dim(m, dim - 1)) {
    u32 const* soe = ask_down(m, dim, dim - 1);
    oup* eos = ask_up(m, dim - 1, dim);
    for (u32 i = 0; i < ne; ++i)
      for (u32 j = 0; j < spe; ++j) {
        u32 s = soe[i * spe + j];
        u32 k;
        out[i * spe + j] = INV;
        for (k = eos->offs[s]; k < eos->offs[s + 1]; ++k)
          if (eos->adj[k] != i) {
            out[i * spe + j] = eos->adj[k];
            break;
          }
      }
  } else {
    u32 const* voe = ask_down(m, dim, 0);
    oup* eov = ask_up(m, 0, dim);
    u32 vpe = DEG[dim][0], vps = DEG[dim - 1][0];
    u32 cap = 64;
    u32* buf = NEW(u32, cap);
    for (u32 i = 0; i < ne; ++i)
      for (u32 j = 0; j < spe; ++j) {
        u32 n = 0;
        for (u32 k = 0; k < vps; ++k) {
          u32 v = voe[i * vpe + co(dim, dim - 1, 0, j, k)];
          u32 f = eov->offs[v], e = eov->offs[v + 1];
          if (k) {
            u32 nn = 0;
            for (u32 a = 0; a < n; ++a)
              if (has_u32(eov->adj + f, e - f, buf[a])) buf[nn++] = buf[a];
            n = nn;
          } else {
            if (e - f > cap) {
              cap = e - f;
              buf = (u32*)realloc(buf, sizeof(u32) * cap);
            }
            for (u32 a = f; a < e; ++a)
              if (eov->adj[a] != i) buf[n++] = eov->adj[a];
          }
        }
        out[i * spe + j] = n ? buf[0] : INV;
      }
    free(buf);
  }
  m->dual = out;
  return out;
}

/* ------------------------------------------------------------------------ */
/* geometry: size.hpp, quality.hpp, algebra.hpp                              */

static void sub3(double const* a, double const* b, double* c)
{
  for (u32 i = 0; i < 3; ++i) c[i] = a[i] - b[i];
}

static void cross3(double const* a, double const* b, double* c)
{
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

static double dot3(double const* a, double const* b)
{
  double d = 0;
  for (u32 i = 0; i < 3; ++i) d += a[i] * b[i];
  return d;
}

static double norm3(double const* a) { return sqrt(dot3(a, a)); }

static double sqdist3(double const* a, double const* b)
{
  double s = 0;
  for (u32 i = 0; i < 3; ++i) {
    double dc = a[i] - b[i];
    s += dc * dc;
  }
  return s;
}

/* triangle_area (size.hpp:14-23) */
static double tri_area(double x[][3])
{
  double v0[3], v1[3], c[3];
  sub3(x[1], x[0], v0);
  sub3(x[2], x[0], v1);
  cross3(v0, v1, c);
  return norm3(c) / 2.0;
}

static double tri_z_area(double x[][3])
{
  double v0[3], v1[3], c[3];
  sub3(x[1], x[0], v0);
  sub3(x[2], x[0], v1);
  cross3(v0, v1, c);
  return c[2] / 2.0;
}

/* tet_volume (size.hpp:36-46) */
static double tet_volume(double x[][3])
{
  double v0[3], v1[3], v2[3], c[3];
  sub3(x[1], x[0], v0);
  sub3(x[2], x[0], v1);
  sub3(x[3], x[0], v2);
  cross3(v0, v1, c);
  return dot3(c, v2) / 6.0;
}

static double measure_entity(u32 dim, double x[][3])
{
  if (dim == 3) return tet_volume(x);
  if (dim == 2) return tri_area(x);
  if (dim == 1) return sqrt(sqdist3(x[1], x[0]));
  return 0.0;
}

static double perfect_tri(void) { return sqrt(3.0) / 4.0; }

static double perfect_tet(void)
{
  double s = sqrt(perfect_tri());
  return (sqrt(2.0) / 12.0) / (s * s * s);
}

/* triangle_quality (quality.hpp:34-47) */
static double tri_quality(double x[][3], int z_area)
{
  double sum = 0;
  for (u32 i = 0; i < 3; ++i) sum += sqdist3(x[i], x[(i + 1) % 3]);
  double lrms = sqrt(sum / 3);
  double a = z_area ? tri_z_area(x) : tri_area(x);
  double q = a / (lrms * lrms);
  return q / perfect_tri();
}

/* tet_quality (quality.hpp:68-89) */
static double tet_quality(double x[][3])
{
  double sum_asq = 0;
  for (u32 i = 0; i < 4; ++i) {
    double t[3][3];
    for (u32 j = 0; j < 3; ++j) memcpy(t[j], x[TET_FV[i][j]], sizeof(t[j]));
    double a = tri_area(t);
    sum_asq += a * a;
  }
  double arms = sqrt(sum_asq / 4.);
  double v = tet_volume(x);
  double r = sqrt(arms);
  double q = v / (r * r * r);
  return q / perfect_tet();
}

/* entity_quality / element_quality (quality.hpp:91-109) */
static double entity_quality(u32 dim, double x[][3])
{
  return dim == 3 ? tet_quality(x) : tri_quality(x, 0);
}
static double element_quality(u32 dim, double x[][3])
{
  return dim == 3 ? tet_quality(x) : tri_quality(x, 1);
}

static void gather_x(double const* coords, u32 const* verts, u32 n,
    double x[][3])
{
  for (u32 j = 0; j < n; ++j) memcpy(x[j], coords + verts[j] * 3, sizeof(x[j]));
}

/* element_qualities (quality.cpp:28-45) */
static double* element_qualities(omesh* m)
{
  u32 dim = m->dim, ne = count(m, dim);
  double* q = NEW(double, ne);
  if (dim < 2) {
    for (u32 i = 0; i < ne; ++i) q[i] = 1.0;
    return q;
  }
  u32 const* voe = ask_down(m, dim, 0);
  double const* x = coords_of(m);
  u32 vpe = DEG[dim][0];
  for (u32 i = 0; i < ne; ++i) {
    double ex[4][3];
    gather_x(x, voe + i * vpe, vpe, ex);
    q[i] = element_quality(dim, ex);
  }
  return q;
}

/* mesh_min_quality (quality.cpp:67-73), minimum over every element */
static double min_quality(omesh* m)
{
  u32 ne = count(m, m->dim);
  double* q = element_qualities(m);
  double mq = DBL_MAX;
  for (u32 i = 0; i < ne; ++i)
    if (q[i] < mq) mq = q[i];
  free(q);
  return mq;
}

/* element_sizes (size.cpp:14-41) */
static double* element_sizes(omesh* m)
{
  u32 dim = m->dim, ne = count(m, dim), vpe = DEG[dim][0];
  u32 const* voe = ask_down(m, dim, 0);
  double const* x = coords_of(m);
  double* s = NEW(double, ne);
  for (u32 i = 0; i < ne; ++i) {
    double ex[4][3];
    gather_x(x, voe + i * vpe, vpe, ex);
    s[i] = measure_entity(dim, ex);
  }
  return s;
}

/* measure_edge (size.cpp:57-69) */
static double* measure_edges(omesh* m)
{
  u32 ne = count(m, 1);
  u32 const* voe = ask_down(m, 1, 0);
  double const* x = coords_of(m);
  double const* h = (double const*)tags_find(&m->tags[0], "adapt_size")->data;
  double* out = NEW(double, ne);
  for (u32 i = 0; i < ne; ++i) {
    u32 a = voe[i * 2], b = voe[i * 2 + 1];
    double len = sqrt(sqdist3(x + b * 3, x + a * 3));
    double want = (h[a] + h[b]) / 2;
    out[i] = len / want;
  }
  return out;
}

/* average_element_field (element_field.hpp:9-25) */
static void average_field(u32 n, u32 const* verts, double const* f, u32 nc,
    double* out)
{
  for (u32 i = 0; i < nc; ++i) out[i] = 0;
  for (u32 i = 0; i < n; ++i)
    for (u32 j = 0; j < nc; ++j) out[j] += f[verts[i] * nc + j];
  for (u32 i = 0; i < nc; ++i) out[i] /= n;
}

/* ------------------------------------------------------------------------ */
/* parallel (single-rank) global numbering: inherit_globals                  */
/* (parallel_modify.cpp:79-111). On one rank every entity is owned, so the   */
/* new numbering is the rank among surviving entities, new ones appended.    */

static void inherit_globals(omesh* m_out, u32 dim, u32 nout)
{
  u64* g = NEW(u64, nout);
  for (u32 i = 0; i < nout; ++i) g[i] = i;
  free(m_out->globals[dim]);
  m_out->globals[dim] = g;
}

/* ------------------------------------------------------------------------ */
/* marking (mark.cpp)                                                        */

static u32* mark_down(omesh* m, u32 high, u32 low, u32 const* marked_highs)
{
  u32 nl = count(m, low);
  oup* u = ask_up(m, low, high);
  u32* out = NEW(u32, nl);
  for (u32 i = 0; i < nl; ++i) {
    out[i] = 0;
    for (u32 j = u->offs[i]; j < u->offs[i + 1]; ++j)
      if (marked_highs[u->adj[j]]) {
        out[i] = 1;
        break;
      }
  }
  return out;
}

static u32* mark_up(omesh* m, u32 low, u32 high, u32 const* marked_lows)
{
  u32 nh = count(m, high), lph = DEG[high][low];
  u32 const* loh = ask_down(m, high, low);
  u32* out = NEW(u32, nh);
  for (u32 i = 0; i < nh; ++i) {
    out[i] = 0;
    for (u32 j = 0; j < lph; ++j)
      if (marked_lows[loh[i * lph + j]]) {
        out[i] = 1;
        break;
      }
  }
  return out;
}

/* mesh_mark_slivers + mesh_mark_dual_layers (mark.cpp:101-147,218-243) */
static u32* mark_slivers(omesh* m, double good_qual, u32 nlayers)
{
  u32 dim = m->dim, ne = count(m, dim), deg = DEG[dim][dim - 1];
  double* q = element_qualities(m);
  u32* s = NEW(u32, ne);
  for (u32 i = 0; i < ne; ++i) s[i] = (q[i] < good_qual) ? 1 : 0;
  free(q);
  u32 const* dual = ask_dual(m);
  for (u32 l = 0; l < nlayers; ++l) {
    u32* o = NEW(u32, ne);
    for (u32 i = 0; i < ne; ++i) {
      o[i] = s[i];
      for (u32 j = 0; j < deg; ++j) {
        u32 e = dual[i * deg + j];
        if (e != INV && s[e]) o[i] = 1;
      }
    }
    free(s);
    s = o;
  }
  return s;
}

/* mesh_unmark_boundary (mark.cpp:198-216) */
static void unmark_boundary(omesh* m, u32 dim, u32* marked)
{
  u32 const* cd = (u32 const*)tags_find(&m->tags[dim], "class_dim")->data;
  u32 n = count(m, dim);
  for (u32 i = 0; i < n; ++i)
    if (cd[i] != m->dim) marked[i] = 0;
}

/* ------------------------------------------------------------------------ */
/* independent set (indset.cpp:55-139)                                       */

static u32* find_indset(omesh* m, u32 ent_dim, u32 const* filter,
    double const* good)
{
  u32 n = count(m, ent_dim);
  ograph* g = ask_star(m, ent_dim, m->dim);
  u64* iota = 0;
  u64 const* glob = m->parallel ? m->globals[ent_dim] : 0;
  if (!glob) {
    iota = NEW(u64, n);
    for (u32 i = 0; i < n; ++i) iota[i] = i;
    glob = iota;
  }
  u32* state = NEW(u32, n);
  for (u32 i = 0; i < n; ++i) state[i] = filter[i] ? UNKNOWN : NOT_IN_SET;
  u32* old = NEW(u32, n);
  int done = 0;
  for (u32 it = 0; it < MAX_ITERATIONS && !done; ++it) {
    memcpy(old, state, sizeof(u32) * n);
    for (u32 i = 0; i < n; ++i) {
      if (old[i] != UNKNOWN) continue;
      u32 f = g->offs[i], e = g->offs[i + 1], j;
      for (j = f; j < e; ++j)
        if (old[g->adj[j]] == IN_SET) break;
      if (j < e) {
        state[i] = NOT_IN_SET;
        continue;
      }
      double myg = good[i];
      for (j = f; j < e; ++j) {
        u32 o = g->adj[j];
        if (old[o] == NOT_IN_SET) continue;
        double og = good[o];
        if (myg == og && glob[o] < glob[i]) break;
        if (myg < og) break;
      }
      if (j == e) state[i] = IN_SET;
    }
    if (u32_max(state, n) < UNKNOWN) done = 1;
  }
  free(old);
  free(iota);
  if (!done) {
    free(state);
    m->err = E_NOCONVERGE;
    return 0;
  }
  return state;
}

/* ------------------------------------------------------------------------ */
/* class inheritance (inherit.cpp:104-232)                                   */

static u32 prods_per_dom(u32 dom, u32 src, u32 prod)
{
  /* get_prods_per_dom (refine_topology.cpp:110-120) */
  if (prod == 0) return dom == src ? 1 : 0;
  u32 base = prod - 1;
  u32 o = dom - 1 - base;
  if (src < o) return 0;
  return DEG[src][o];
}

typedef struct {
  u32 ndoms[4];
  u32* pdo[4]; /* prods_of_doms_offsets, 0 when a domain dim gives nothing */
  int own[4];  /* which pdo arrays this struct owns */
} odoms;

static void doms_free(odoms* d)
{
  for (u32 i = 0; i < 4; ++i)
    if (d->own[i]) free(d->pdo[i]);
}

static void ngen_offsets(odoms const* d, u32 ngo[5])
{
  ngo[0] = 0;
  for (u32 i = 0; i < 4; ++i) {
    u32 n = (d->ndoms[i] && d->pdo[i]) ? d->pdo[i][d->ndoms[i]] : 0;
    ngo[i + 1] = ngo[i] + n;
  }
}

static void inherit_u32_tag(omesh* m, omesh* m_out, u32 prod, odoms const* d,
    char const* name)
{
  otag* t = tags_find(&m->tags[prod], name);
  u32 nc = t->ncomps;
  u32 const* dom_data[4] = {0, 0, 0, 0};
  dom_data[0] = (u32 const*)t->data;
  for (u32 k = 1; k <= m->dim; ++k) {
    otag* tk = tags_find(&m->tags[k], name);
    dom_data[k] = tk ? (u32 const*)tk->data : 0;
  }
  u32 ngo[5];
  ngen_offsets(d, ngo);
  u32* out = NEW(u32, ngo[4] * nc);
  for (u32 k = 0; k < 4; ++k) {
    if (!(d->ndoms[k] && dom_data[k] && d->pdo[k])) continue;
    u32* g = (u32*)expand_bytes(dom_data[k], d->pdo[k], d->ndoms[k], nc, 4);
    memcpy(out + ngo[k] * nc, g, sizeof(u32) * (ngo[k + 1] - ngo[k]) * nc);
    free(g);
  }
  tags_add(&m_out->tags[prod], T_U32, t->name, nc, X_NOT, out);
}

static void inherit_class(omesh* m, omesh* m_out, u32 prod, odoms const* d)
{
  if (!tags_find(&m->tags[0], "class_dim")) return;
  inherit_u32_tag(m, m_out, prod, d, "class_dim");
  if (tags_find(&m->tags[0], "class_id"))
    inherit_u32_tag(m, m_out, prod, d, "class_id");
}

/* concat_verts_of_ents (inherit.cpp:234-255) */
static u32* concat_verts(u32 dim, u32 n, u32 const* voe, u32 const* same_offs,
    u32 ngen, u32 const* gen_verts, u32* p_nout)
{
  u32 vpe = DEG[dim][0];
  u32 nsame = same_offs[n];
  u32* out = NEW(u32, (nsame + ngen) * vpe);
  u32* s = (u32*)expand_bytes(voe, same_offs, n, vpe, 4);
  memcpy(out, s, sizeof(u32) * nsame * vpe);
  free(s);
  memcpy(out + nsame * vpe, gen_verts, sizeof(u32) * ngen * vpe);
  *p_nout = nsame + ngen;
  return out;
}

/* interp_to_elems of "coordinates" (element_field.cpp:27-51) */
static void interp_coords_to_elems(omesh* m)
{
  u32 dim = m->dim, ne = count(m, dim), vpe = DEG[dim][0];
  u32 const* voe = ask_down(m, dim, 0);
  double const* x = coords_of(m);
  double* out = NEW(double, ne * 3);
  for (u32 i = 0; i < ne; ++i) average_field(vpe, voe + i * vpe, x, 3, out + i * 3);
  tags_add(&m->tags[dim], T_F64, "coordinates", 3, X_NOT, out);
}

/* ------------------------------------------------------------------------ */
/* refinement (refine.cpp, refine_common.cpp, refine_qualities.cpp,          */
/* splits_to_domains.cpp, refine_topology.cpp, refine_nodal.cpp,             */
/* refine_conserve.cpp, refine_fit.cpp)                                      */

/* refine_quality (refine_qualities.cpp:16-82), src_dim 1, require_better 0 */
static double* refine_qualities(omesh* m, u32* cand, double qual_floor)
{
  u32 dim = m->dim, ne = count(m, 1);
  double* q = NEW(double, ne);
  for (u32 i = 0; i < ne; ++i) q[i] = 0.0;
  if (dim < 2) {
    for (u32 i = 0; i < ne; ++i) q[i] = 1.0;
    return q;
  }
  u32 const* vos = ask_down(m, 1, 0);
  u32 const* voe = ask_down(m, dim, 0);
  oup* eos = ask_up(m, 1, dim);
  double const* x = coords_of(m);
  u32 vpe = DEG[dim][0];
  for (u32 i = 0; i < ne; ++i) {
    if (!cand[i]) continue;
    double split[3];
    average_field(2, vos + i * 2, x, 3, split);
    double minq = 1;
    for (u32 j = eos->offs[i]; j < eos->offs[i + 1]; ++j) {
      u32 dir = eos->dirs[j], e = eos->adj[j];
      for (u32 k = 0; k < 2; ++k) {
        u32 o = co(dim, 1, 0, dir, k);
        u32 base = opp(dim, 0, o);
        double ex[4][3];
        for (u32 l = 0; l < vpe - 1; ++l)
          memcpy(ex[l], x + voe[e * vpe + co(dim, dim - 1, 0, base, l)] * 3,
              sizeof(ex[l]));
        memcpy(ex[vpe - 1], split, sizeof(split));
        double qq = entity_quality(dim, ex);
        if (qq < minq) minq = qq;
      }
    }
    if (minq < qual_floor)
      cand[i] = 0;
    else
      q[i] = minq;
  }
  return q;
}

typedef struct {
  u32* offset;    /* exscan of which domains split, n+1 */
  u32* direction; /* local index of the split source in the domain */
  u32* vert;      /* generated vertex of the split source */
} osplits;

/* refine_verts (refine_common.cpp:29-54) */
static void refine_verts(omesh* m, omesh* m_out, u32 const* gen_offs)
{
  u32 nv = count(m, 0), ns = count(m, 1), nsplit = gen_offs[ns];
  u32 nv_out = nv + nsplit;
  set_ents(m_out, 0, nv_out, 0);
  u32 const* vos = ask_down(m, 1, 0);
  for (u32 t = 0; t < m->tags[0].n; ++t) {
    otag* tg = m->tags[0].at[t];
    if (tg->type != T_F64) continue;
    u32 nc = tg->ncomps;
    double* out = NEW(double, (size_t)nv_out * nc);
    memcpy(out, tg->data, sizeof(double) * nv * nc);
    double const* f = (double const*)tg->data;
    for (u32 i = 0; i < ns; ++i) {
      if (gen_offs[i] == gen_offs[i + 1]) continue;
      average_field(2, vos + i * 2, f, nc, out + (size_t)(nv + gen_offs[i]) * nc);
    }
    tags_add(&m_out->tags[0], T_F64, tg->name, nc, X_NOT, out);
  }
  if (m->parallel) inherit_globals(m_out, 0, nv_out);
}

static void refine_ents(omesh* m, omesh* m_out, u32 const* gen_offs)
{
  u32 dim = m->dim, src = 1;
  u32 ns = count(m, src), nv = count(m, 0);
  u32* gen_vert = NEW(u32, ns);
  for (u32 i = 0; i < ns; ++i)
    gen_vert[i] = (gen_offs[i] != gen_offs[i + 1]) ? nv + gen_offs[i] : INV;
  osplits sp[4];
  memset(sp, 0, sizeof(sp));
  sp[0].offset = u32_filled(nv + 1, 0);
  for (u32 dd = 1; dd <= dim; ++dd) {
    if (!has_dim(m, dd)) continue;
    u32 nd = count(m, dd);
    if (dd < src) {
      sp[dd].offset = u32_filled(nd + 1, 0);
      continue;
    }
    /* split_to_domain (splits_to_domains.cpp:13-31) */
    u32 spd = DEG[dd][src];
    u32 const* sod = ask_down(m, dd, src);
    u32* will = u32_filled(nd, 0);
    sp[dd].direction = u32_filled(nd, INV);
    sp[dd].vert = u32_filled(nd, INV);
    for (u32 i = 0; i < nd; ++i)
      for (u32 j = 0; j < spd; ++j) {
        u32 s = sod[i * spd + j];
        if (gen_offs[s] == gen_offs[s + 1]) continue;
        will[i] = 1;
        sp[dd].direction[i] = j;
        sp[dd].vert[i] = gen_vert[s];
        break;
      }
    sp[dd].offset = u32_exscan(will, nd);
    free(will);
  }
  free(gen_vert);
  for (u32 prod = 0; prod <= dim; ++prod) {
    if (!m->full && 0 < prod && prod < dim) continue;
    /* setup_refine (inherit.cpp:104-138) */
    odoms d;
    memset(&d, 0, sizeof(d));
    u32 np = count(m, prod);
    d.ndoms[0] = np;
    d.pdo[0] = negate_offsets(sp[prod].offset, np);
    d.own[0] = 1;
    u32 first = 1, last = dim;
    if (m->full) {
      first = (src > prod) ? src : prod;
    } else {
      first = last = (prod == 0) ? src : dim;
    }
    for (u32 dd = first; dd <= last; ++dd) {
      d.ndoms[dd] = count(m, dd);
      u32 ppd = prods_per_dom(dd, src, prod);
      d.pdo[dd] = NEW(u32, d.ndoms[dd] + 1);
      for (u32 i = 0; i <= d.ndoms[dd]; ++i) d.pdo[dd][i] = sp[dd].offset[i] * ppd;
      d.own[dd] = 1;
    }
    u32 ngo[5];
    ngen_offsets(&d, ngo);
    if (prod) {
      u32 vpp = DEG[prod][0], nout = ngo[4];
      u32* vop = NEW(u32, (size_t)nout * vpp);
      u32* same = (u32*)expand_bytes(ask_down(m, prod, 0), d.pdo[0], np, vpp, 4);
      memcpy(vop, same, sizeof(u32) * d.pdo[0][np] * vpp);
      free(same);
      for (u32 dd = 1; dd <= dim; ++dd) {
        if (!(d.ndoms[dd] && d.pdo[dd])) continue;
        /* refine_topology / refine_domain_entity (refine_topology.cpp:26-107) */
        u32 base_dim = prod - 1;
        u32 opp_dim = dd - 1 - base_dim;
        if (src < opp_dim) continue;
        u32 ops = DEG[src][opp_dim];
        u32 nd = d.ndoms[dd];
        if (!sp[dd].offset[nd]) continue;
        u32 vpd = DEG[dd][0], vpb = vpp - 1;
        u32 const* vod = ask_down(m, dd, 0);
        u32* outp = vop + (size_t)ngo[dd] * vpp;
        for (u32 i = 0; i < nd; ++i) {
          if (sp[dd].offset[i] == sp[dd].offset[i + 1]) continue;
          u32 dir = sp[dd].direction[i];
          u32* p = outp + (size_t)sp[dd].offset[i] * ops * vpp;
          for (u32 j = 0; j < ops; ++j) {
            u32 o = co(dd, src, opp_dim, dir, j);
            u32 b = opp(dd, opp_dim, o);
            for (u32 k = 0; k < vpb; ++k)
              p[k] = vod[i * vpd + co(dd, base_dim, 0, b, k)];
            p[vpb] = sp[dd].vert[i];
            p += vpp;
          }
        }
      }
      set_ents(m_out, prod, nout, vop);
      if (m->parallel) inherit_globals(m_out, prod, nout);
    }
    inherit_class(m, m_out, prod, &d);
    if (prod == dim) {
      /* refine_conserve then refine_fit (refine_conserve.cpp, refine_fit.cpp) */
      for (int pass = 0; pass < 2; ++pass) {
        u32 want = pass == 0 ? X_CONSERVE : X_POINTWISE;
        for (u32 t = 0; t < m->tags[dim].n; ++t) {
          otag* tg = m->tags[dim].at[t];
          if (tg->type != T_F64 || tg->transfer != want) continue;
          u32 nc = tg->ncomps, ne = count(m, dim);
          double const* in = (double const*)tg->data;
          double* out = NEW(double, (size_t)ngo[4] * nc);
          double* s = (double*)expand_bytes(in, d.pdo[0], ne, nc, 8);
          memcpy(out, s, sizeof(double) * d.pdo[0][ne] * nc);
          free(s);
          u32 const* po = d.pdo[dim];
          double* g = out + (size_t)ngo[dim] * nc;
          for (u32 i = 0; i < ne; ++i) {
            u32 f = po[i], e = po[i + 1];
            double denom = e - f;
            for (u32 j = f; j < e; ++j)
              for (u32 k = 0; k < nc; ++k)
                g[j * nc + k] = pass == 0 ? in[i * nc + k] / denom : in[i * nc + k];
          }
          tags_add(&m_out->tags[dim], T_F64, tg->name, nc, tg->transfer, out);
        }
      }
    }
    doms_free(&d);
  }
  for (u32 dd = 0; dd <= dim; ++dd) {
    free(sp[dd].offset);
    free(sp[dd].direction);
    free(sp[dd].vert);
  }
}

/* refine_common (refine_common.cpp:162-190), src_dim 1 */
static u32 refine_common(omesh* m, u32* cand, double qual_floor)
{
  u32 ne = count(m, 1);
  if (!u32_max(cand, ne)) return 0;
  double* q = refine_qualities(m, cand, qual_floor);
  if (!u32_max(cand, ne)) {
    free(q);
    return 0;
  }
  u32* indset = find_indset(m, 1, cand, q);
  free(q);
  if (!indset) return 0;
  u32* gen_offs = u32_exscan(indset, ne);
  free(indset);
  omesh* m_out = mesh_new(m->dim, m->full, m->parallel);
  refine_verts(m, m_out, gen_offs);
  refine_ents(m, m_out, gen_offs);
  free(gen_offs);
  mesh_overwrite(m, m_out);
  return 1;
}

/* refine_by_size (refine.cpp:17-27) */
static u32 refine_by_size(omesh* m, double qual_floor)
{
  u32 ne = count(m, 1);
  double* len = measure_edges(m);
  u32* cand = NEW(u32, ne);
  for (u32 i = 0; i < ne; ++i) cand[i] = len[i] > 1.0;
  free(len);
  u32 r = refine_common(m, cand, qual_floor);
  free(cand);
  return r;
}

/* uniformly_refine (refine.cpp:29-35) */
static void uniformly_refine(omesh* m)
{
  u32 ne = count(m, 1);
  u32* cand = u32_filled(ne, 1);
  refine_common(m, cand, 0.0);
  free(cand);
}

/* ------------------------------------------------------------------------ */
/* coarsening (coarsen.cpp, coarsen_common.cpp, check_collapse_class.cpp,    */
/* coarsen_qualities.cpp, collapses_to_verts.cpp, collapses_to_ents.cpp,     */
/* coarsen_topology.cpp, coarsen_conserve.cpp, coarsen_fit.cpp, qr.cpp)      */

static u32 collapses(u32 code, u32 dir) { return (code & (1u << dir)) != 0; }

/* check_collapse_class (check_collapse_class.cpp:12-147) */
static void check_collapse_class(omesh* m, u32* codes)
{
  u32 ne = count(m, 1), dim = m->dim;
  u32 const* voe = ask_down(m, 1, 0);
  u32 const* cdv = (u32 const*)tags_find(&m->tags[0], "class_dim")->data;
  u32 const* cde = (u32 const*)tags_find(&m->tags[1], "class_dim")->data;
  for (u32 i = 0; i < ne; ++i) {
    if (codes[i] == DONT_COLLAPSE) continue;
    u32 c[3] = {cdv[voe[i * 2]], cdv[voe[i * 2 + 1]], cde[i]};
    if (c[0] == c[1]) {
      if (c[0] != c[2]) codes[i] = DONT_COLLAPSE;
      continue;
    }
    for (u32 j = 0; j < 2; ++j) {
      if (!collapses(codes[i], j)) continue;
      if (c[j] != c[2]) codes[i] &= ~(1u << j);
    }
  }
  for (u32 ed = 2; ed <= dim; ++ed) {
    oup* u = ask_up(m, 1, ed);
    u32 const* vot = ask_down(m, ed, 0);
    u32 const* sot = ask_down(m, ed, ed - 1);
    u32 vpt = DEG[ed][0], spt = DEG[ed][ed - 1];
    u32 const* cdt = (u32 const*)tags_find(&m->tags[ed], "class_dim")->data;
    u32 const* cds = (u32 const*)tags_find(&m->tags[ed - 1], "class_dim")->data;
    for (u32 i = 0; i < ne; ++i) {
      if (codes[i] == DONT_COLLAPSE) continue;
      for (u32 j = u->offs[i]; j < u->offs[i + 1]; ++j) {
        u32 t = u->adj[j], dir = u->dirs[j];
        for (u32 k = 0; k < 2; ++k) {
          if (!collapses(codes[i], k)) continue;
          u32 va = voe[i * 2 + (1 - k)];
          for (u32 l = 0; l < 2; ++l) {
            u32 eev = co(ed, 1, 0, dir, l);
            if (vot[t * vpt + eev] == va) {
              u32 side = sot[t * spt + opp(ed, 0, eev)];
              if (cds[side] != cdt[t]) codes[i] &= ~(1u << k);
              break;
            }
          }
        }
      }
    }
  }
}

/* coarsen_quality (coarsen_qualities.cpp:12-79); out is 2 per edge */
static double* coarsen_qualities(omesh* m, u32* codes, double floor_q,
    double const* elem_quals)
{
  u32 dim = m->dim, ne = count(m, 1);
  double* out = NEW(double, ne * 2);
  for (u32 i = 0; i < ne * 2; ++i) out[i] = 0.0;
  if (dim < 2) {
    for (u32 i = 0; i < ne * 2; ++i) out[i] = 1.0;
    return out;
  }
  u32 vpe = DEG[dim][0];
  u32 const* voe = ask_down(m, dim, 0);
  u32 const* vos = ask_down(m, 1, 0);
  oup* eov = ask_up(m, 0, dim);
  double const* x = coords_of(m);
  for (u32 i = 0; i < ne; ++i) {
    if (codes[i] == DONT_COLLAPSE) continue;
    for (u32 j = 0; j < 2; ++j) {
      if (!collapses(codes[i], j)) continue;
      double minq = 1, old_minq = 1;
      u32 col = vos[i * 2 + j], gen = vos[i * 2 + 1 - j];
      double ex[4][3];
      memcpy(ex[vpe - 1], x + gen * 3, sizeof(ex[0]));
      for (u32 k = eov->offs[col]; k < eov->offs[col + 1]; ++k) {
        u32 e = eov->adj[k];
        u32 const* ve = voe + e * vpe;
        int adjacent = 0;
        if (elem_quals && elem_quals[e] < old_minq) old_minq = elem_quals[e];
        for (u32 l = 0; l < vpe; ++l)
          if (ve[l] == gen) adjacent = 1;
        if (adjacent) continue;
        u32 base = opp(dim, 0, eov->dirs[k]);
        for (u32 l = 0; l < vpe - 1; ++l)
          memcpy(ex[l], x + ve[co(dim, dim - 1, 0, base, l)] * 3, sizeof(ex[0]));
        double q = element_quality(dim, ex);
        if (q < minq) minq = q;
      }
      if (minq < floor_q || (elem_quals && minq <= old_minq))
        codes[i] &= ~(1u << j);
      else
        out[i * 2 + j] = minq;
    }
  }
  return out;
}

/* collapse_to_vert (collapses_to_verts.cpp:13-42) */
static void collapses_to_verts(omesh* m, u32 const* codes, double const* q2,
    u32* cand, double* col_qual)
{
  u32 nv = count(m, 0);
  oup* u = ask_up(m, 0, 1);
  for (u32 i = 0; i < nv; ++i) {
    double maxq = 0;
    u32 c = 0;
    for (u32 j = u->offs[i]; j < u->offs[i + 1]; ++j) {
      u32 e = u->adj[j], d = u->dirs[j];
      if (!collapses(codes[e], d)) continue;
      double q = q2[e * 2 + d];
      if (!c) {
        c = 1;
        maxq = q;
      } else if (q > maxq) {
        maxq = q;
      }
    }
    cand[i] = c;
    col_qual[i] = c ? maxq : 0.0;
  }
}

/* vertex_dest (collapses_to_verts.cpp:72-105) */
static u32* vertex_destinations(omesh* m, u32 const* indset, u32 const* codes,
    double const* q2, double const* col_qual)
{
  u32 nv = count(m, 0);
  oup* u = ask_up(m, 0, 1);
  u32 const* vos = ask_down(m, 1, 0);
  u32* out = u32_filled(nv, INV);
  for (u32 i = 0; i < nv; ++i) {
    if (!indset[i]) continue;
    double maxq = col_qual[i];
    if (maxq == 1e10) maxq = -1e10;
    for (u32 j = u->offs[i]; j < u->offs[i + 1]; ++j) {
      u32 e = u->adj[j], d = u->dirs[j];
      if (!collapses(codes[e], d)) continue;
      double q = q2[e * 2 + d];
      if (q == 1e10) q = -1e10;
      if (q == maxq) {
        out[i] = vos[e * 2 + (1 - d)];
        break;
      }
    }
  }
  return out;
}

/* ---- QR least squares used by coarsen_fit (qr.cpp:42-205) ---- */
static double sgn(double x) { return (x < 0) ? -1 : 1; }
static double sq(double x) { return x * x; }

static u32 get_reflector2(double a[MAX_PTS][4], double v[MAX_PTS], u32 k,
    u32 npts)
{
  double cnorm = 0;
  for (u32 i = k; i < npts; ++i) cnorm += sq(a[i][k]);
  cnorm = sqrt(cnorm);
  if (cnorm < 1e-6) return 0;
  for (u32 i = 0; i < k; ++i) v[i] = 0;
  for (u32 i = k; i < npts; ++i) v[i] = a[i][k];
  v[k] += sgn(a[k][k]) * cnorm;
  double rnorm = 0;
  for (u32 i = k; i < npts; ++i) rnorm += sq(v[i]);
  rnorm = sqrt(rnorm);
  for (u32 i = k; i < npts; ++i) v[i] /= rnorm;
  return 1;
}

static u32 qr_decomp2(double a[MAX_PTS][4], double q[MAX_PTS][MAX_PTS],
    double r[MAX_PTS][4], u32 npts)
{
  for (u32 i = 0; i < npts; ++i)
    for (u32 j = 0; j < 4; ++j) r[i][j] = a[i][j];
  for (u32 i = 0; i < npts; ++i)
    for (u32 j = 0; j < npts; ++j) q[i][j] = (double)(i == j);
  double v[MAX_PTS];
  memset(v, 0, sizeof(v));
  u32 rank = 0;
  for (u32 k = 0; k < 4; ++k)
    if (get_reflector2(r, v, k, npts)) {
      for (u32 j = 0; j < 4; ++j) {
        double dot = 0;
        for (u32 i = k; i < npts; ++i) dot += r[i][j] * v[i];
        for (u32 i = k; i < npts; ++i) r[i][j] -= 2 * dot * v[i];
      }
      for (u32 i = 0; i < npts; ++i) {
        double dot = 0;
        for (u32 j = k; j < npts; ++j) dot += q[i][j] * v[j];
        for (u32 j = k; j < npts; ++j) q[i][j] -= 2 * dot * v[j];
      }
      ++rank;
    }
  return rank;
}

static void qr_solve2(double q[MAX_PTS][MAX_PTS], double r[MAX_PTS][4],
    double b[MAX_PTS], u32 npts, double x[4])
{
  double y[4];
  for (u32 i = 0; i < 4; ++i) {
    y[i] = 0;
    for (u32 j = 0; j < npts; ++j) y[i] += q[j][i] * b[j];
  }
  for (u32 ii = 0; ii < 4; ++ii) {
    u32 i = 4 - ii - 1;
    x[i] = y[i];
    for (u32 j = i + 1; j < 4; ++j) x[i] -= r[i][j] * x[j];
    x[i] /= r[i][i];
  }
}

/* coarsen_conserve / coarsen_fit on the element tags of m_out */
static void coarsen_transfer(omesh* m, omesh* m_out, u32 const* gen_offs_v,
    u32 const* gen_offs_e, u32 const* same_offs_e)
{
  u32 dim = m->dim, nv = count(m, 0), ne = count(m, dim);
  oup* eov = ask_up(m, 0, dim);
  u32 nsame = same_offs_e[ne], ngen = gen_offs_e[ne];
  /* coarsen_conserve (coarsen_conserve.cpp:15-137) */
  int any_f64 = 0;
  for (u32 t = 0; t < m->tags[dim].n; ++t)
    if (m->tags[dim].at[t]->type == T_F64) any_f64 = 1;
  if (any_f64) {
    double* sizes = element_sizes(m_out);
    for (u32 t = 0; t < m->tags[dim].n; ++t) {
      otag* tg = m->tags[dim].at[t];
      if (tg->type != T_F64 || tg->transfer != X_CONSERVE) continue;
      u32 nc = tg->ncomps;
      double const* in = (double const*)tg->data;
      double* out = NEW(double, (size_t)(nsame + ngen) * nc);
      double* s = (double*)expand_bytes(in, same_offs_e, ne, nc, 8);
      memcpy(out, s, sizeof(double) * nsame * nc);
      free(s);
      double* g = out + (size_t)nsame * nc;
      for (u32 i = 0; i < nv; ++i) {
        if (gen_offs_v[i] == gen_offs_v[i + 1]) continue;
        u32 f = eov->offs[i], e = eov->offs[i + 1];
        double sum[MAX_NCOMPS];
        for (u32 k = 0; k < nc; ++k) sum[k] = 0;
        for (u32 j = f; j < e; ++j)
          for (u32 k = 0; k < nc; ++k) sum[k] = sum[k] + in[eov->adj[j] * nc + k];
        double cav = 0;
        for (u32 j = f; j < e; ++j) {
          u32 el = eov->adj[j];
          if (gen_offs_e[el] == gen_offs_e[el + 1]) continue;
          cav += sizes[gen_offs_e[el] + nsame];
        }
        for (u32 j = f; j < e; ++j) {
          u32 el = eov->adj[j];
          if (gen_offs_e[el] == gen_offs_e[el + 1]) continue;
          u32 ge = gen_offs_e[el];
          double sc = sizes[ge + nsame] / cav;
          for (u32 k = 0; k < nc; ++k) g[ge * nc + k] = sum[k] * sc;
        }
      }
      tags_add(&m_out->tags[dim], T_F64, tg->name, nc, tg->transfer, out);
    }
    free(sizes);
  }
  /* coarsen_fit (coarsen_fit.cpp:17-185) */
  int any_fit = 0;
  for (u32 t = 0; t < m->tags[dim].n; ++t)
    if (m->tags[dim].at[t]->type == T_F64 &&
        m->tags[dim].at[t]->transfer == X_POINTWISE)
      any_fit = 1;
  if (!any_fit) return;
  if (!tags_find(&m->tags[dim], "coordinates")) interp_coords_to_elems(m);
  interp_coords_to_elems(m_out);
  double const* oldx = (double const*)tags_find(&m->tags[dim], "coordinates")->data;
  double const* newx = (double const*)tags_find(&m_out->tags[dim], "coordinates")->data;
  for (u32 t = 0; t < m->tags[dim].n; ++t) {
    otag* tg = m->tags[dim].at[t];
    if (tg->type != T_F64 || tg->transfer != X_POINTWISE) continue;
    u32 nc = tg->ncomps;
    double const* in = (double const*)tg->data;
    double* out = NEW(double, (size_t)(nsame + ngen) * nc);
    double* s = (double*)expand_bytes(in, same_offs_e, ne, nc, 8);
    memcpy(out, s, sizeof(double) * nsame * nc);
    free(s);
    double* g = out + (size_t)nsame * nc;
    for (u32 i = 0; i < nv; ++i) {
      if (gen_offs_v[i] == gen_offs_v[i + 1]) continue;
      u32 f = eov->offs[i], e = eov->offs[i + 1];
      u32 npts = e - f;
      if (npts > MAX_PTS) npts = MAX_PTS;
      int fit = npts >= 4;
      double q[MAX_PTS][MAX_PTS];
      double r[MAX_PTS][4];
      if (fit) {
        double a[MAX_PTS][4];
        for (u32 j = 0; j < npts; ++j) {
          u32 oe = eov->adj[f + j];
          a[j][0] = 1.0;
          memcpy(&a[j][1], oldx + 3 * oe, sizeof(double) * 3);
        }
        if (qr_decomp2(a, q, r, npts) < 4) fit = 0;
      }
      for (u32 j = 0; j < nc; ++j) {
        double b[MAX_PTS], c[4], avg = 0;
        if (fit) {
          for (u32 k = 0; k < npts; ++k) b[k] = in[eov->adj[f + k] * nc + j];
          qr_solve2(q, r, b, npts, c);
        } else {
          avg = 0;
          for (u32 k = f; k < e; ++k) avg += in[eov->adj[k] * nc + j];
          avg /= (e - f);
        }
        for (u32 k = f; k < e; ++k) {
          u32 oe = eov->adj[k];
          if (gen_offs_e[oe] == gen_offs_e[oe + 1]) continue;
          u32 ge = gen_offs_e[oe];
          if (fit) {
            double dd = dot3(c + 1, newx + (ge + nsame) * 3);
            g[ge * nc + j] = c[0] + dd;
          } else {
            g[ge * nc + j] = avg;
          }
        }
      }
    }
    tags_add(&m_out->tags[dim], T_F64, tg->name, nc, tg->transfer, out);
  }
}

/* coarsen_ents (coarsen_common.cpp:35-89) for one entity dimension */
static void coarsen_ents(omesh* m, omesh* m_out, u32 ed, u32 const* gen_offs_v,
    u32 const* gen_vert_v, u32 const* same_offs_v, u32 const* fused_ents,
    u32** p_fused_sides)
{
  u32 n = count(m, ed), vpe = DEG[ed][0], spe = DEG[ed][ed - 1];
  u32 const* voe = ask_down(m, ed, 0);
  u32 const* soe = ask_down(m, ed, ed - 1);
  u32* fused = u32_filled(count(m, ed - 1), 0);
  u32* will_gen = u32_filled(n, 0);
  u32* gen_vert = u32_filled(n, INV);
  u32* gen_dir = u32_filled(n, INV);
  u32* is_same = NEW(u32, n);
  /* collapse_to_ent (collapses_to_ents.cpp:11-64) */
  for (u32 i = 0; i < n; ++i) {
    u32 const* v = voe + i * vpe;
    u32 col = INV, dir = INV;
    for (u32 j = 0; j < vpe; ++j)
      if (gen_offs_v[v[j]] != gen_offs_v[v[j] + 1]) {
        col = v[j];
        dir = j;
      }
    if (dir == INV) {
      is_same[i] = 1;
      continue;
    }
    is_same[i] = 0;
    u32 gv = gen_vert_v[col], gd = INV;
    for (u32 j = 0; j < vpe; ++j)
      if (v[j] == gv) gd = j;
    if (gd != INV) {
      fused[soe[i * spe + opp(ed, 0, gd)]] = 1;
      continue;
    }
    if (!(fused_ents && fused_ents[i])) {
      will_gen[i] = 1;
      gen_vert[i] = gv;
      gen_dir[i] = dir;
    }
  }
  u32* gen_offs = u32_exscan(will_gen, n);
  u32* same_offs = u32_exscan(is_same, n);
  free(will_gen);
  free(is_same);
  /* coarsen_elem (coarsen_topology.cpp:9-34) */
  u32 ngen = gen_offs[n];
  u32* gv = NEW(u32, (size_t)ngen * vpe);
  for (u32 i = 0; i < n; ++i) {
    if (gen_offs[i] == gen_offs[i + 1]) continue;
    u32* o = gv + (size_t)gen_offs[i] * vpe;
    u32 b = opp(ed, 0, gen_dir[i]);
    for (u32 j = 0; j < vpe - 1; ++j) o[j] = voe[i * vpe + co(ed, ed - 1, 0, b, j)];
    o[vpe - 1] = gen_vert[i];
  }
  free(gen_vert);
  free(gen_dir);
  u32 nout;
  u32* out = concat_verts(ed, n, voe, same_offs, ngen, gv, &nout);
  free(gv);
  for (u32 i = 0; i < nout * vpe; ++i) out[i] = same_offs_v[out[i]];
  set_ents(m_out, ed, nout, out);
  /* setup_coarsen (inherit.cpp:140-157) */
  odoms d;
  memset(&d, 0, sizeof(d));
  d.ndoms[0] = n;
  d.pdo[0] = same_offs;
  d.ndoms[ed] = n;
  d.pdo[ed] = gen_offs;
  inherit_class(m, m_out, ed, &d);
  if (m->parallel) inherit_globals(m_out, ed, nout);
  if (ed == m->dim) coarsen_transfer(m, m_out, gen_offs_v, gen_offs, same_offs);
  free(gen_offs);
  free(same_offs);
  *p_fused_sides = fused;
}

/* coarsen_common (coarsen_common.cpp:109-239) */
static u32 coarsen_common(omesh* m, u32* codes, double qual_floor,
    int require_better)
{
  u32 ne = count(m, 1), nv = count(m, 0), dim = m->dim;
  if (u32_max(codes, ne) == DONT_COLLAPSE) return 0;
  check_collapse_class(m, codes);
  if (u32_max(codes, ne) == DONT_COLLAPSE) return 0;
  double* eq = require_better ? element_qualities(m) : 0;
  double* q2 = coarsen_qualities(m, codes, qual_floor, eq);
  free(eq);
  if (u32_max(codes, ne) == DONT_COLLAPSE) {
    free(q2);
    return 0;
  }
  u32* cand = NEW(u32, nv);
  double* cq = NEW(double, nv);
  collapses_to_verts(m, codes, q2, cand, cq);
  u32* indset = find_indset(m, 0, cand, cq);
  free(cand);
  if (!indset) {
    free(cq);
    free(q2);
    return 0;
  }
  /* coarsen_interior (coarsen_common.cpp:191-219) */
  u32* gen_vert = vertex_destinations(m, indset, codes, q2, cq);
  free(cq);
  free(q2);
  u32* gen_offs_v = u32_exscan(indset, nv);
  free(indset);
  u32* same_offs_v = negate_offsets(gen_offs_v, nv);
  u32 nv_out = same_offs_v[nv];
  omesh* m_out = mesh_new(dim, m->full, m->parallel);
  set_ents(m_out, 0, nv_out, 0);
  /* tags_subset (subset.cpp:15-43) */
  for (u32 t = 0; t < m->tags[0].n; ++t) {
    otag* tg = m->tags[0].at[t];
    void* o = expand_bytes(tg->data, same_offs_v, nv, tg->ncomps, tag_esz(tg->type));
    tags_add(&m_out->tags[0], tg->type, tg->name, tg->ncomps, tg->transfer, o);
  }
  if (m->parallel) inherit_globals(m_out, 0, nv_out);
  u32* fused[4] = {0, 0, 0, 0};
  for (u32 dd = 0; dd < dim; ++dd) {
    u32 d = dim - dd;
    coarsen_ents(m, m_out, d, gen_offs_v, gen_vert, same_offs_v, fused[d],
        &fused[d - 1]);
  }
  for (u32 d = 0; d < 4; ++d) free(fused[d]);
  free(gen_vert);
  free(gen_offs_v);
  free(same_offs_v);
  mesh_overwrite(m, m_out);
  return 1;
}

/* coarsen_by_size (coarsen.cpp:23-36) */
static u32 coarsen_by_size(omesh* m, double qual_floor, double size_floor)
{
  u32 ne = count(m, 1);
  double* len = measure_edges(m);
  u32* codes = NEW(u32, ne);
  for (u32 i = 0; i < ne; ++i)
    codes[i] = (len[i] < size_floor) ? COLLAPSE_BOTH : DONT_COLLAPSE;
  free(len);
  u32 r = coarsen_common(m, codes, qual_floor, 0);
  free(codes);
  return r;
}

/* coarsen_slivers (coarsen.cpp:51-70) */
static u32 coarsen_slivers(omesh* m, double qual_floor, u32 nlayers)
{
  u32 dim = m->dim, ne = count(m, 1);
  u32* sl = mark_slivers(m, qual_floor, nlayers);
  u32* mv = mark_down(m, dim, 0, sl);
  free(sl);
  u32 const* voe = ask_down(m, 1, 0);
  u32* codes = NEW(u32, ne);
  for (u32 i = 0; i < ne; ++i) {
    codes[i] = 0;
    for (u32 j = 0; j < 2; ++j)
      if (mv[voe[i * 2 + j]]) codes[i] |= 1u << j;
  }
  free(mv);
  u32 r = coarsen_common(m, codes, 0.0, 1);
  free(codes);
  return r;
}

/* ------------------------------------------------------------------------ */
/* edge swapping (swap.cpp, swap_qualities.cpp, edge_ring.cpp,               */
/* edge_swap.cpp, swap_topology.cpp, swap_conserve.cpp, swap_fit.cpp)        */

typedef struct {
  u32 ntri[MAX_EDGE_SWAP + 1];            /* triangles per triangulation */
  u32 nmesh[MAX_EDGE_SWAP + 1];           /* triangulations per ring size */
  u32 tri[MAX_EDGE_SWAP + 1][42][5][3];   /* ring-vertex triples */
  u32 uniq[MAX_EDGE_SWAP + 1][42][5];     /* cache slot of each triangle */
  u32 nint[MAX_EDGE_SWAP + 1];            /* interior edges per triangulation */
  u32 iedge[MAX_EDGE_SWAP + 1][42][4][2]; /* interior edges */
} swap_tables;

static swap_tables ST;
static int st_ready = 0;

/* interior edges of a polygon triangulation, in the order the reference's
   own side derivation emits them (test_print_swap_edges.cpp:29-58): for each
   triangle in order, each side (0,1),(1,2),(2,0) whose neighbour triangle
   has a larger index. */
static void swap_tables_init(void)
{
  if (st_ready) return;
  memset(&ST, 0, sizeof(ST));
  for (u32 n = 3; n <= MAX_EDGE_SWAP; ++n) {
    char const* s = oracle_polygon_triangulations[n];
    u32 nt = n - 2, nm = 0, uniq_n = 0;
    u32 seen[64][3];
    while (*s) {
      for (u32 t = 0; t < nt; ++t) {
        for (u32 k = 0; k < 3; ++k) ST.tri[n][nm][t][k] = (u32)(s[k] - '0');
        s += 3;
        if (*s == '.') ++s;
        u32 a;
        for (a = 0; a < uniq_n; ++a)
          if (!memcmp(seen[a], ST.tri[n][nm][t], sizeof(seen[a]))) break;
        if (a == uniq_n) memcpy(seen[uniq_n++], ST.tri[n][nm][t], sizeof(seen[a]));
        ST.uniq[n][nm][t] = a;
      }
      while (*s == ' ') ++s;
      ++nm;
    }
    ST.ntri[n] = nt;
    ST.nmesh[n] = nm;
    for (u32 mm = 0; mm < nm; ++mm) {
      u32 ni = 0;
      for (u32 t = 0; t < nt; ++t)
        for (u32 j = 0; j < 3; ++j) {
          u32 a = ST.tri[n][mm][t][j], b = ST.tri[n][mm][t][(j + 1) % 3];
          /* neighbour across side (a,b): the first other triangle with both */
          u32 nb = INV;
          for (u32 o = 0; o < nt && nb == INV; ++o) {
            if (o == t) continue;
            int ha = 0, hb = 0;
            for (u32 k = 0; k < 3; ++k) {
              ha |= ST.tri[n][mm][o][k] == a;
              hb |= ST.tri[n][mm][o][k] == b;
            }
            if (ha && hb) nb = o;
          }
          if (nb != INV && t < nb) {
            ST.iedge[n][mm][ni][0] = a;
            ST.iedge[n][mm][ni][1] = b;
            ++ni;
          }
        }
      ST.nint[n] = ni;
    }
  }
  st_ready = 1;
}

/* find_edge_ring (edge_ring.cpp:12-74) */
static u32 find_edge_ring(u32 edge, oup const* toe, u32 const* voe,
    u32 const* vot, u32* edge_v, u32* ring_v)
{
  u32 f = toe->offs[edge], e = toe->offs[edge + 1];
  u32 rs = e - f;
  if (rs > MAX_EDGE_SWAP) return rs;
  edge_v[0] = voe[edge * 2];
  edge_v[1] = voe[edge * 2 + 1];
  u32 ta[MAX_EDGE_SWAP], tb[MAX_EDGE_SWAP];
  for (u32 i = f; i < e; ++i) {
    u32 t = toe->adj[i], te = toe->dirs[i];
    u32 const* tv = vot + t * 4;
    u32 align = (tv[TET_EV[te][0]] != edge_v[0]) ? 1 : 0;
    u32 o = OPP_RE[te];
    ta[i - f] = tv[TET_EV[o][align ^ 0]];
    tb[i - f] = tv[TET_EV[o][align ^ 1]];
  }
  for (u32 i = 0; i + 1 < rs; ++i) {
    u32 j;
    for (j = i + 1; j < rs; ++j)
      if (ta[j] == tb[i]) break;
    if (j == rs) return INV; /* malformed ring */
    u32 xa = ta[j], xb = tb[j];
    ta[j] = ta[i + 1];
    tb[j] = tb[i + 1];
    ta[i + 1] = xa;
    tb[i + 1] = xb;
  }
  for (u32 i = 0; i < rs; ++i) ring_v[i] = ta[i];
  return rs;
}

/* choose_edge_swap (edge_swap.cpp:230-280) */
static void choose_edge_swap(u32 rs, double ex[2][3], double rx[][3],
    u32* p_code, double* p_q)
{
  unsigned char cached[64];
  double cache[64];
  memset(cached, 0, sizeof(cached));
  u32 code = INV;
  double best = -1;
  for (u32 i = 0; i < ST.nmesh[rs]; ++i) {
    double mesh_minq = 1;
    for (u32 j = 0; j < ST.ntri[rs]; ++j) {
      u32 slot = ST.uniq[rs][i][j];
      if (!cached[slot]) {
        double tx[4][3];
        for (u32 k = 0; k < 3; ++k) memcpy(tx[k], rx[ST.tri[rs][i][j][k]], sizeof(tx[k]));
        double tri_minq = 1;
        for (u32 k = 0; k < 2; ++k) {
          memcpy(tx[3], ex[1 - k], sizeof(tx[3]));
          double q = tet_quality(tx);
          if (q < tri_minq) tri_minq = q;
          double tmp[3];
          memcpy(tmp, tx[0], sizeof(tmp));
          memcpy(tx[0], tx[1], sizeof(tmp));
          memcpy(tx[1], tmp, sizeof(tmp));
        }
        cached[slot] = 1;
        cache[slot] = tri_minq;
      }
      double tq = cache[slot];
      if (tq < mesh_minq) mesh_minq = tq;
      if (mesh_minq < 0) break;
    }
    if (mesh_minq > best) {
      code = i;
      best = mesh_minq;
    }
  }
  *p_code = code;
  *p_q = best;
}

/* swap_quality (swap_qualities.cpp:13-61) */
static void swap_qualities(omesh* m, u32* cand, double* quals, u32* rsz)
{
  u32 ne = count(m, 1);
  oup* toe = ask_up(m, 1, 3);
  u32 const* voe = ask_down(m, 1, 0);
  u32 const* vot = ask_down(m, 3, 0);
  double const* x = coords_of(m);
  double* eq = element_qualities(m);
  for (u32 i = 0; i < ne; ++i) {
    quals[i] = 0;
    rsz[i] = 0;
    if (!cand[i]) continue;
    double old_minq = 1;
    for (u32 j = toe->offs[i]; j < toe->offs[i + 1]; ++j)
      if (eq[toe->adj[j]] < old_minq) old_minq = eq[toe->adj[j]];
    u32 ev[2], rv[MAX_EDGE_SWAP];
    u32 rs = find_edge_ring(i, toe, voe, vot, ev, rv);
    if (rs > MAX_EDGE_SWAP) {
      cand[i] = 0;
      continue;
    }
    double ex[2][3], rx[MAX_EDGE_SWAP][3];
    memcpy(ex[0], x + ev[0] * 3, sizeof(ex[0]));
    memcpy(ex[1], x + ev[1] * 3, sizeof(ex[1]));
    for (u32 j = 0; j < rs; ++j) memcpy(rx[j], x + rv[j] * 3, sizeof(rx[j]));
    u32 code;
    double q;
    choose_edge_swap(rs, ex, rx, &code, &q);
    if (q > old_minq) {
      quals[i] = q;
      rsz[i] = rs;
    } else {
      cand[i] = 0;
    }
  }
  free(eq);
}

/* count_swap_ents (edge_swap.cpp:375-386) */
static u32 count_swap_ents(u32 rs, u32 dim)
{
  if (dim == 1) return ST.nint[rs];
  if (dim == 2) return ST.ntri[rs] + 2 * ST.nint[rs];
  return 2 * ST.ntri[rs];
}

/* get_swap_ents (edge_swap.cpp:282-373) */
static void get_swap_ents(u32 rs, u32 code, u32 dim, u32 const* ev,
    u32 const* rv, u32* out)
{
  if (dim == 1) {
    for (u32 i = 0; i < ST.nint[rs]; ++i)
      for (u32 j = 0; j < 2; ++j) out[i * 2 + j] = rv[ST.iedge[rs][code][i][j]];
  } else if (dim == 2) {
    u32 ni = ST.nint[rs];
    for (u32 i = 0; i < ni; ++i)
      for (u32 j = 0; j < 2; ++j) {
        for (u32 k = 0; k < 2; ++k) out[i * 6 + j * 3 + k] = rv[ST.iedge[rs][code][i][k]];
        out[i * 6 + j * 3 + 2] = ev[j];
      }
    out += ni * 6;
    for (u32 i = 0; i < ST.ntri[rs]; ++i)
      for (u32 j = 0; j < 3; ++j) out[i * 3 + j] = rv[ST.tri[rs][code][i][j]];
  } else {
    for (u32 i = 0; i < ST.ntri[rs]; ++i) {
      u32 tv[4];
      for (u32 j = 0; j < 3; ++j) tv[j] = rv[ST.tri[rs][code][i][j]];
      for (u32 j = 0; j < 2; ++j) {
        tv[3] = ev[1 - j];
        for (u32 k = 0; k < 4; ++k) *out++ = tv[k];
        u32 t = tv[0];
        tv[0] = tv[1];
        tv[1] = t;
      }
    }
  }
}

/* swap_ents (swap.cpp:27-69) */
static void swap_ents(omesh* m, omesh* m_out, u32 ed, u32 const* indset,
    u32 const* rsz)
{
  u32 ne = count(m, 1), n = count(m, ed), vpe = DEG[ed][0];
  u32* cnt = NEW(u32, ne);
  for (u32 i = 0; i < ne; ++i) cnt[i] = indset[i] ? count_swap_ents(rsz[i], ed) : 0;
  u32* gen_offs = u32_exscan(cnt, ne);
  free(cnt);
  u32 ngen = gen_offs[ne];
  /* swap_cavity (swap_topology.cpp:42-71) re-derives each chosen swap */
  oup* toe = ask_up(m, 1, 3);
  u32 const* voe1 = ask_down(m, 1, 0);
  u32 const* vot = ask_down(m, 3, 0);
  double const* x = coords_of(m);
  u32* gv = NEW(u32, (size_t)ngen * vpe);
  for (u32 i = 0; i < ne; ++i) {
    if (!indset[i]) continue;
    u32 ev[2], rv[MAX_EDGE_SWAP];
    u32 rs = find_edge_ring(i, toe, voe1, vot, ev, rv);
    double ex[2][3], rx[MAX_EDGE_SWAP][3];
    memcpy(ex[0], x + ev[0] * 3, sizeof(ex[0]));
    memcpy(ex[1], x + ev[1] * 3, sizeof(ex[1]));
    for (u32 j = 0; j < rs; ++j) memcpy(rx[j], x + rv[j] * 3, sizeof(rx[j]));
    u32 code;
    double q;
    choose_edge_swap(rs, ex, rx, &code, &q);
    get_swap_ents(rs, code, ed, ev, rv, gv + (size_t)gen_offs[i] * vpe);
  }
  u32* old = mark_up(m, 1, ed, indset);
  for (u32 i = 0; i < n; ++i) old[i] = !old[i];
  u32* same_offs = u32_exscan(old, n);
  free(old);
  u32 nout;
  u32* out = concat_verts(ed, n, ask_down(m, ed, 0), same_offs, ngen, gv, &nout);
  free(gv);
  set_ents(m_out, ed, nout, out);
  if (m->full) {
    /* setup_swap (inherit.cpp:159-175) */
    odoms d;
    memset(&d, 0, sizeof(d));
    d.ndoms[0] = n;
    d.pdo[0] = same_offs;
    d.ndoms[1] = ne;
    d.pdo[1] = gen_offs;
    inherit_class(m, m_out, ed, &d);
  }
  if (m->parallel) inherit_globals(m_out, ed, nout);
  if (ed == m->dim) {
    u32 nsame = same_offs[n];
    int any_f64 = 0;
    for (u32 t = 0; t < m->tags[ed].n; ++t)
      if (m->tags[ed].at[t]->type == T_F64) any_f64 = 1;
    oup* eoe = ask_up(m, 1, ed);
    if (any_f64) {
      /* swap_conserve (swap_conserve.cpp:15-129) */
      double* sizes = element_sizes(m_out);
      for (u32 t = 0; t < m->tags[ed].n; ++t) {
        otag* tg = m->tags[ed].at[t];
        if (tg->type != T_F64 || tg->transfer != X_CONSERVE) continue;
        u32 nc = tg->ncomps;
        double const* in = (double const*)tg->data;
        double* o = NEW(double, (size_t)(nsame + ngen) * nc);
        double* s = (double*)expand_bytes(in, same_offs, n, nc, 8);
        memcpy(o, s, sizeof(double) * nsame * nc);
        free(s);
        double* g = o + (size_t)nsame * nc;
        for (u32 i = 0; i < ne; ++i) {
          if (gen_offs[i] == gen_offs[i + 1]) continue;
          double sum[MAX_NCOMPS];
          for (u32 k = 0; k < nc; ++k) sum[k] = 0;
          for (u32 j = eoe->offs[i]; j < eoe->offs[i + 1]; ++j)
            for (u32 k = 0; k < nc; ++k) sum[k] = sum[k] + in[eoe->adj[j] * nc + k];
          double cav = 0;
          for (u32 j = gen_offs[i]; j < gen_offs[i + 1]; ++j) cav += sizes[nsame + j];
          for (u32 j = gen_offs[i]; j < gen_offs[i + 1]; ++j) {
            double sc = sizes[nsame + j] / cav;
            for (u32 k = 0; k < nc; ++k) g[j * nc + k] = sum[k] * sc;
          }
        }
        tags_add(&m_out->tags[ed], T_F64, tg->name, nc, tg->transfer, o);
      }
      free(sizes);
    }
    /* swap_fit (swap_fit.cpp:24-125): plain average over the old cavity */
    for (u32 t = 0; t < m->tags[ed].n; ++t) {
      otag* tg = m->tags[ed].at[t];
      if (tg->type != T_F64 || tg->transfer != X_POINTWISE) continue;
      u32 nc = tg->ncomps;
      double const* in = (double const*)tg->data;
      double* o = NEW(double, (size_t)(nsame + ngen) * nc);
      double* s = (double*)expand_bytes(in, same_offs, n, nc, 8);
      memcpy(o, s, sizeof(double) * nsame * nc);
      free(s);
      double* g = o + (size_t)nsame * nc;
      for (u32 i = 0; i < ne; ++i) {
        if (gen_offs[i] == gen_offs[i + 1]) continue;
        u32 f = eoe->offs[i], e = eoe->offs[i + 1];
        for (u32 j = 0; j < nc; ++j) {
          double avg = 0;
          for (u32 k = f; k < e; ++k) avg += in[eoe->adj[k] * nc + j];
          avg /= (e - f);
          for (u32 ge = gen_offs[i]; ge < gen_offs[i + 1]; ++ge) g[ge * nc + j] = avg;
        }
      }
      tags_add(&m_out->tags[ed], T_F64, tg->name, nc, tg->transfer, o);
    }
  }
  free(gen_offs);
  free(same_offs);
}

/* swap_slivers + swap_common + swap_interior (swap.cpp:71-154) */
static u32 swap_slivers(omesh* m, double good_qual, u32 nlayers)
{
  if (m->dim != 3) {
    m->err = E_BAD;
    return 0;
  }
  swap_tables_init();
  u32 ne = count(m, 1), dim = m->dim;
  u32* sl = mark_slivers(m, good_qual, nlayers);
  u32* cand = mark_down(m, dim, 1, sl);
  free(sl);
  if (!u32_max(cand, ne)) {
    free(cand);
    return 0;
  }
  unmark_boundary(m, 1, cand);
  if (!u32_max(cand, ne)) {
    free(cand);
    return 0;
  }
  double* q = NEW(double, ne);
  u32* rsz = NEW(u32, ne);
  swap_qualities(m, cand, q, rsz);
  if (!u32_max(cand, ne)) {
    free(cand);
    free(q);
    free(rsz);
    return 0;
  }
  u32* indset = find_indset(m, 1, cand, q);
  free(cand);
  free(q);
  if (!indset) {
    free(rsz);
    return 0;
  }
  u32 nv = count(m, 0);
  omesh* m_out = mesh_new(dim, m->full, m->parallel);
  set_ents(m_out, 0, nv, 0);
  for (u32 t = 0; t < m->tags[0].n; ++t) {
    otag* tg = m->tags[0].at[t];
    size_t bytes = (size_t)nv * tg->ncomps * tag_esz(tg->type);
    void* o = xmalloc(bytes);
    memcpy(o, tg->data, bytes);
    tags_add(&m_out->tags[0], tg->type, tg->name, tg->ncomps, tg->transfer, o);
  }
  if (m->parallel && m->globals[0]) {
    m_out->globals[0] = NEW(u64, nv);
    memcpy(m_out->globals[0], m->globals[0], sizeof(u64) * nv);
  }
  if (!m->full)
    swap_ents(m, m_out, dim, indset, rsz);
  else
    for (u32 d = 1; d <= dim; ++d) swap_ents(m, m_out, d, indset, rsz);
  free(indset);
  free(rsz);
  mesh_overwrite(m, m_out);
  return 1;
}

/* ------------------------------------------------------------------------ */
/* adapt driver (adapt.cpp:36-94)                                            */

static u32 adapt(omesh* m, double size_floor, double good_qual, u32 nlayers,
    u32 max_ops)
{
  u32 ops = 0;
#define INCR()                  \
  do {                          \
    if (ops > max_ops) {        \
      m->err = E_MAXOPS;        \
      return ops > 0;           \
    }                           \
    ++ops;                      \
  } while (0)
  double qf = min_quality(m);
  if (good_qual < qf) qf = good_qual;
  while (refine_by_size(m, qf)) INCR();
  if (m->err) return ops > 0;
  while (coarsen_by_size(m, qf, size_floor)) INCR();
  if (m->err) return ops > 0;
  for (;;) {
    double prev = min_quality(m);
    if (prev >= good_qual) break;
    if (m->dim == 3 && swap_slivers(m, good_qual, nlayers)) {
      INCR();
      continue;
    }
    if (m->err) break;
    if (coarsen_slivers(m, good_qual, nlayers)) {
      INCR();
      continue;
    }
    break;
  }
#undef INCR
  return ops > 0;
}

/* ------------------------------------------------------------------------ */
/* classification (derive_model.cpp:218-448, bfs.cpp)                        */

static void derive_model(omesh* m, double crease)
{
  u32 dim = m->dim;
  u32 nel = count(m, dim);
  tags_add(&m->tags[dim], T_U32, "class_dim", 1, X_NOT, u32_filled(nel, dim));
  u32 ns = count(m, dim - 1);
  oup* eos = ask_up(m, dim - 1, dim);
  u32* bside = NEW(u32, ns);
  for (u32 i = 0; i < ns; ++i) bside[i] = (eos->offs[i + 1] - eos->offs[i]) < 2;
  u32* scd = NEW(u32, ns);
  for (u32 i = 0; i < ns; ++i) scd[i] = dim - bside[i];
  tags_add(&m->tags[dim - 1], T_U32, "class_dim", 1, X_NOT, scd);
  if (dim >= 2) {
    double const* x = coords_of(m);
    u32 const* vos = ask_down(m, dim - 1, 0);
    double* nrm = NEW(double, 3 * ns);
    for (u32 i = 0; i < ns; ++i) {
      if (!bside[i]) continue;
      double* nn = nrm + i * 3;
      if (dim - 1 == 1) {
        sub3(x + vos[i * 2 + 1] * 3, x + vos[i * 2] * 3, nn);
      } else {
        double b0[3], b1[3];
        sub3(x + vos[i * 3 + 1] * 3, x + vos[i * 3] * 3, b0);
        sub3(x + vos[i * 3 + 2] * 3, x + vos[i * 3] * 3, b1);
        cross3(b0, b1, nn);
      }
      double s = 1.0 / norm3(nn);
      for (u32 k = 0; k < 3; ++k) nn[k] = nn[k] * s;
    }
    u32 nh = count(m, dim - 2);
    u32* bh = mark_down(m, dim - 1, dim - 2, bside);
    oup* soh = ask_up(m, dim - 2, dim - 1);
    u32* crease_h = NEW(u32, nh);
    for (u32 i = 0; i < nh; ++i) {
      double ang = 0;
      if (bh[i]) {
        u32 adj[2] = {0, 0}, na = 0;
        for (u32 j = soh->offs[i]; j < soh->offs[i + 1]; ++j)
          if (bside[soh->adj[j]] && na < 2) adj[na++] = soh->adj[j];
        ang = acos(dot3(nrm + adj[0] * 3, nrm + adj[1] * 3));
      }
      crease_h[i] = ang > crease;
    }
    free(nrm);
    u32* hcd = NEW(u32, nh);
    for (u32 i = 0; i < nh; ++i) hcd[i] = dim - bh[i] - crease_h[i];
    free(bh);
    tags_add(&m->tags[dim - 2], T_U32, "class_dim", 1, X_NOT, hcd);
    if (dim == 3) {
      u32 nv = count(m, 0);
      oup* eov = ask_up(m, 0, 1);
      u32* vcd = NEW(u32, nv);
      for (u32 i = 0; i < nv; ++i) {
        u32 nin = 0, d = 3;
        for (u32 j = eov->offs[i]; j < eov->offs[i + 1]; ++j) {
          u32 e = eov->adj[j];
          if (crease_h[e]) ++nin;
          if (hcd[e] < d) d = hcd[e];
        }
        vcd[i] = d - (nin > 2);
      }
      tags_add(&m->tags[0], T_U32, "class_dim", 1, X_NOT, vcd);
    }
    free(crease_h);
  }
  free(bside);
  /* mesh_derive_class_id (derive_model.cpp:414-442) */
  {
    u32 nv = count(m, 0);
    u32 const* vcd = (u32 const*)tags_find(&m->tags[0], "class_dim")->data;
    u32* vid = u32_filled(nv, INV);
    u32 k = 0;
    for (u32 i = 0; i < nv; ++i)
      if (vcd[i] == 0) vid[i] = k++;
    tags_add(&m->tags[0], T_U32, "class_id", 1, X_NOT, vid);
  }
  for (u32 d = 1; d <= dim; ++d) {
    /* set_equal_order_class_id (derive_model.cpp:318-390): components of the
       entities classified on dimension d, connected through sides that are
       also classified on d, numbered by their smallest member. */
    u32 n = count(m, d);
    u32 const* cd = (u32 const*)tags_find(&m->tags[d], "class_dim")->data;
    u32 const* cds = (u32 const*)tags_find(&m->tags[d - 1], "class_dim")->data;
    u32 const* sod = ask_down(m, d, d - 1);
    oup* dos = ask_up(m, d - 1, d);
    u32 spd = DEG[d][d - 1];
    u32* id = u32_filled(n, INV);
    u32* queue = NEW(u32, n);
    u32 comp = 0;
    for (u32 i = 0; i < n; ++i) {
      if (cd[i] != d || id[i] != INV) continue;
      u32 b = 0, e = 0;
      queue[e++] = i;
      id[i] = comp;
      while (b != e) {
        u32 u = queue[b++];
        for (u32 j = 0; j < spd; ++j) {
          u32 s = sod[u * spd + j];
          if (cds[s] != d) continue;
          for (u32 l = dos->offs[s]; l < dos->offs[s + 1]; ++l) {
            u32 o = dos->adj[l];
            if (o == u || cd[o] != d) continue;
            if (id[o] == INV) {
              id[o] = comp;
              queue[e++] = o;
            }
            break;
          }
        }
      }
      ++comp;
    }
    free(queue);
    tags_add(&m->tags[d], T_U32, "class_id", 1, X_NOT, id);
  }
  for (u32 dd = 1; dd <= dim; ++dd) {
    /* project_class_id_onto (derive_model.cpp:392-412) */
    u32 d = dim - dd, nl = count(m, d);
    oup* u = ask_up(m, d, d + 1);
    u32 const* hcd = (u32 const*)tags_find(&m->tags[d + 1], "class_dim")->data;
    u32 const* hid = (u32 const*)tags_find(&m->tags[d + 1], "class_id")->data;
    u32 const* lcd = (u32 const*)tags_find(&m->tags[d], "class_dim")->data;
    u32* lid = (u32*)tags_find(&m->tags[d], "class_id")->data;
    for (u32 i = 0; i < nl; ++i)
      for (u32 j = u->offs[i]; j < u->offs[i + 1]; ++j)
        if (hcd[u->adj[j]] == lcd[i]) lid[i] = hid[u->adj[j]];
  }
}

/* ------------------------------------------------------------------------ */
/* seeded synthetic inputs                                                   */

static u64 splitmix64(u64* s)
{
  u64 z = (*s += 0x9E3779B97F4A7C15ul);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ul;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBul;
  return z ^ (z >> 31);
}

static double unit_draw(u64* s)
{
  return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
}

/* ======================================================================== */
/* exported C interface (used through ctypes by oracle/oracle.py)            */

#define EXPORT __attribute__((visibility("default")))

/* n^3 hexahedra split 6 ways, interior vertices perturbed; center[3] is the
   next draw of the same stream, scaled to [0.3, 0.7]. */
EXPORT void or_box(u32 n, u64 seed, double pert, double* coords, u32* conn,
    double* center)
{
  u32 n1 = n + 1;
  u64 s = seed;
  double amp = pert / (double)n;
  for (u32 k = 0; k < n1; ++k)
    for (u32 j = 0; j < n1; ++j)
      for (u32 i = 0; i < n1; ++i) {
        u32 v = (k * n1 + j) * n1 + i;
        double* x = coords + (size_t)v * 3;
        x[0] = (double)i / (double)n;
        x[1] = (double)j / (double)n;
        x[2] = (double)k / (double)n;
        if (i > 0 && i < n && j > 0 && j < n && k > 0 && k < n)
          for (u32 c = 0; c < 3; ++c) x[c] = x[c] + amp * (2.0 * unit_draw(&s) - 1.0);
      }
  for (u32 c = 0; c < 3; ++c) center[c] = 0.3 + 0.4 * unit_draw(&s);
  for (u32 k = 0; k < n; ++k)
    for (u32 j = 0; j < n; ++j)
      for (u32 i = 0; i < n; ++i) {
        u32 h = (k * n + j) * n + i;
        for (u32 t = 0; t < 6; ++t)
          for (u32 c = 0; c < 4; ++c) {
            u32 const* cc = CUBE_CORNER[CUBE_SPLIT[t][c]];
            conn[(size_t)(h * 6 + t) * 4 + c] =
              ((k + cc[2]) * n1 + (j + cc[1])) * n1 + (i + cc[0]);
          }
      }
}

/* h(x) = h0 + h1 * |x - c| per vertex */
EXPORT void or_radial_size(u32 nverts, double const* coords, double const* c,
    double h0, double h1, double* out)
{
  for (u32 v = 0; v < nverts; ++v) {
    double const* x = coords + (size_t)v * 3;
    double dx = x[0] - c[0], dy = x[1] - c[1], dz = x[2] - c[2];
    out[v] = h0 + h1 * sqrt(dx * dx + dy * dy + dz * dz);
  }
}

EXPORT omesh* or_new_reduced(u32 dim, u32 nverts, double const* coords,
    u32 nelems, u32 const* conn)
{
  omesh* m = mesh_new(dim, 0, 0);
  set_ents(m, 0, nverts, 0);
  u32 vpe = DEG[dim][0];
  u32* c = NEW(u32, (size_t)nelems * vpe);
  memcpy(c, conn, sizeof(u32) * nelems * vpe);
  set_ents(m, dim, nelems, c);
  double* x = NEW(double, (size_t)nverts * 3);
  memcpy(x, coords, sizeof(double) * nverts * 3);
  tags_add(&m->tags[0], T_F64, "coordinates", 3, X_NOT, x);
  return m;
}

EXPORT void or_derive_model_full(omesh* m)
{
  derive_model(m, ORACLE_PI / 4);
  m->full = 1;
}

/* mesh_make_parallel (mesh.cpp:320-327) */
EXPORT void or_make_parallel(omesh* m)
{
  m->parallel = 1;
  for (u32 d = 0; d <= m->dim; ++d)
    if (has_dim(m, d)) inherit_globals(m, d, count(m, d));
}

EXPORT void or_free(omesh* m)
{
  mesh_clear(m);
  free(m);
}

EXPORT u32 or_dim(omesh* m) { return m->dim; }
EXPORT u32 or_count(omesh* m, u32 dim) { return count(m, dim); }
EXPORT int or_error(omesh* m) { return m->err; }

EXPORT void or_add_tag(omesh* m, u32 dim, char const* name, u32 type,
    u32 ncomps, u32 transfer, void const* data)
{
  size_t bytes = (size_t)count(m, dim) * ncomps * tag_esz(type);
  void* d = xmalloc(bytes);
  memcpy(d, data, bytes);
  tags_add(&m->tags[dim], type, name, ncomps, transfer, d);
}

EXPORT void or_free_tag(omesh* m, u32 dim, char const* name)
{
  tags_remove(&m->tags[dim], name);
}

EXPORT u32 or_ntags(omesh* m, u32 dim) { return m->tags[dim].n; }
EXPORT char const* or_tag_name(omesh* m, u32 dim, u32 i) { return m->tags[dim].at[i]->name; }
EXPORT u32 or_tag_type(omesh* m, u32 dim, u32 i) { return m->tags[dim].at[i]->type; }
EXPORT u32 or_tag_ncomps(omesh* m, u32 dim, u32 i) { return m->tags[dim].at[i]->ncomps; }
EXPORT u32 or_tag_transfer(omesh* m, u32 dim, u32 i) { return m->tags[dim].at[i]->transfer; }
EXPORT void or_tag_data(omesh* m, u32 dim, u32 i, void* out)
{
  otag* t = m->tags[dim].at[i];
  memcpy(out, t->data, (size_t)count(m, dim) * t->ncomps * tag_esz(t->type));
}

EXPORT void or_down(omesh* m, u32 high, u32 low, u32* out)
{
  memcpy(out, ask_down(m, high, low), sizeof(u32) * count(m, high) * DEG[high][low]);
}

EXPORT u32 or_up_size(omesh* m, u32 low, u32 high)
{
  return ask_up(m, low, high)->offs[count(m, low)];
}

EXPORT void or_up(omesh* m, u32 low, u32 high, u32* offs, u32* adj, u32* dirs)
{
  oup* u = ask_up(m, low, high);
  u32 n = count(m, low);
  memcpy(offs, u->offs, sizeof(u32) * (n + 1));
  memcpy(adj, u->adj, sizeof(u32) * u->offs[n]);
  memcpy(dirs, u->dirs, sizeof(u32) * u->offs[n]);
}

EXPORT u32 or_star_size(omesh* m, u32 low, u32 high)
{
  return ask_star(m, low, high)->offs[count(m, low)];
}

EXPORT void or_star(omesh* m, u32 low, u32 high, u32* offs, u32* adj)
{
  ograph* g = ask_star(m, low, high);
  u32 n = count(m, low);
  memcpy(offs, g->offs, sizeof(u32) * (n + 1));
  memcpy(adj, g->adj, sizeof(u32) * g->offs[n]);
}

EXPORT void or_dual(omesh* m, u32* out)
{
  u32 d = m->dim;
  memcpy(out, ask_dual(m), sizeof(u32) * count(m, d) * DEG[d][d - 1]);
}

EXPORT u32 or_has_globals(omesh* m, u32 dim)
{
  return m->parallel && m->globals[dim] != 0;
}

EXPORT void or_globals(omesh* m, u32 dim, u64* out)
{
  memcpy(out, m->globals[dim], sizeof(u64) * count(m, dim));
}

EXPORT void or_set_globals(omesh* m, u32 dim, u64 const* in)
{
  u32 n = count(m, dim);
  free(m->globals[dim]);
  m->globals[dim] = NEW(u64, n);
  memcpy(m->globals[dim], in, sizeof(u64) * n);
}

EXPORT double or_min_quality(omesh* m) { return min_quality(m); }

EXPORT void or_qualities(omesh* m, double* out)
{
  double* q = element_qualities(m);
  memcpy(out, q, sizeof(double) * count(m, m->dim));
  free(q);
}

EXPORT void or_edge_lengths(omesh* m, double* out)
{
  double* l = measure_edges(m);
  memcpy(out, l, sizeof(double) * count(m, 1));
  free(l);
}

EXPORT u32 or_refine_by_size(omesh* m, double qf) { return refine_by_size(m, qf); }
EXPORT void or_uniformly_refine(omesh* m) { uniformly_refine(m); }
EXPORT u32 or_coarsen_by_size(omesh* m, double qf, double sf)
{
  return coarsen_by_size(m, qf, sf);
}
EXPORT u32 or_coarsen_slivers(omesh* m, double qf, u32 nl)
{
  return coarsen_slivers(m, qf, nl);
}
EXPORT u32 or_swap_slivers(omesh* m, double gq, u32 nl) { return swap_slivers(m, gq, nl); }
EXPORT u32 or_adapt(omesh* m, double sf, double gq, u32 nl, u32 mo)
{
  return adapt(m, sf, gq, nl, mo);
}

/* per-stage sets, same layout as the reference driver's refd_*_sets */
EXPORT u32 or_refine_sets(omesh* m, double qf, u32* cand, u32* good,
    double* quals, u32* indset)
{
  u32 ne = count(m, 1);
  double* len = measure_edges(m);
  u32* g = NEW(u32, ne);
  for (u32 i = 0; i < ne; ++i) cand[i] = g[i] = len[i] > 1.0;
  free(len);
  double* q = refine_qualities(m, g, qf);
  u32 any = 0;
  for (u32 i = 0; i < ne; ++i) {
    good[i] = g[i];
    quals[i] = g[i] ? q[i] : 0.0;
    indset[i] = 0;
    any |= g[i];
  }
  if (any) {
    u32* s = find_indset(m, 1, g, q);
    if (s) memcpy(indset, s, sizeof(u32) * ne);
    free(s);
  }
  free(g);
  free(q);
  return any;
}

EXPORT u32 or_coarsen_sets(omesh* m, double qf, double sf, u32* codes_size,
    u32* codes_class, u32* codes_qual, double* quals2, u32* cand,
    double* col_qual, u32* indset, u32* gen_vert)
{
  u32 ne = count(m, 1), nv = count(m, 0);
  double* len = measure_edges(m);
  u32* codes = NEW(u32, ne);
  for (u32 i = 0; i < ne; ++i)
    codes[i] = codes_size[i] = (len[i] < sf) ? COLLAPSE_BOTH : DONT_COLLAPSE;
  free(len);
  for (u32 i = 0; i < nv; ++i) {
    cand[i] = 0;
    col_qual[i] = 0;
    indset[i] = 0;
    gen_vert[i] = INV;
  }
  check_collapse_class(m, codes);
  memcpy(codes_class, codes, sizeof(u32) * ne);
  double* q2 = coarsen_qualities(m, codes, qf, 0);
  u32 any = 0;
  for (u32 i = 0; i < ne; ++i) {
    codes_qual[i] = codes[i];
    for (u32 j = 0; j < 2; ++j) quals2[i * 2 + j] = collapses(codes[i], j) ? q2[i * 2 + j] : 0.0;
    any |= codes[i];
  }
  if (!any) {
    free(codes);
    free(q2);
    return 0;
  }
  collapses_to_verts(m, codes, q2, cand, col_qual);
  u32* s = find_indset(m, 0, cand, col_qual);
  if (s) {
    u32* gv = vertex_destinations(m, s, codes, q2, col_qual);
    for (u32 i = 0; i < nv; ++i) {
      indset[i] = s[i];
      gen_vert[i] = s[i] ? gv[i] : INV;
    }
    free(gv);
  }
  free(s);
  free(codes);
  free(q2);
  return 1;
}

EXPORT u32 or_swap_sets(omesh* m, double gq, u32 nl, u32* slivers_out,
    u32* cand, u32* interior, u32* good, double* quals, u32* ring_sizes,
    u32* indset)
{
  swap_tables_init();
  u32 dim = m->dim, ne = count(m, 1), nel = count(m, dim);
  u32* sl = mark_slivers(m, gq, nl);
  memcpy(slivers_out, sl, sizeof(u32) * nel);
  u32* c = mark_down(m, dim, 1, sl);
  free(sl);
  memcpy(cand, c, sizeof(u32) * ne);
  unmark_boundary(m, 1, c);
  memcpy(interior, c, sizeof(u32) * ne);
  for (u32 i = 0; i < ne; ++i) {
    good[i] = 0;
    quals[i] = 0;
    ring_sizes[i] = 0;
    indset[i] = 0;
  }
  if (!u32_max(c, ne)) {
    free(c);
    return 0;
  }
  double* q = NEW(double, ne);
  u32* rs = NEW(u32, ne);
  swap_qualities(m, c, q, rs);
  u32 any = 0;
  for (u32 i = 0; i < ne; ++i) {
    good[i] = c[i];
    if (c[i]) {
      quals[i] = q[i];
      ring_sizes[i] = rs[i];
      any = 1;
    }
  }
  if (any) {
    u32* s = find_indset(m, 1, c, q);
    if (s) memcpy(indset, s, sizeof(u32) * ne);
    free(s);
  }
  free(c);
  free(q);
  free(rs);
  return any;
}

/* polygon-triangulation tables as the swap code sees them, for tests */
EXPORT u32 or_swap_table(u32 rs, u32* ntri, u32* nmesh, u32* nint, u32* tris,
    u32* iedges)
{
  swap_tables_init();
  if (rs < 3 || rs > MAX_EDGE_SWAP) return 0;
  *ntri = ST.ntri[rs];
  *nmesh = ST.nmesh[rs];
  *nint = ST.nint[rs];
  for (u32 i = 0; i < ST.nmesh[rs]; ++i) {
    for (u32 j = 0; j < ST.ntri[rs]; ++j)
      for (u32 k = 0; k < 3; ++k) *tris++ = ST.tri[rs][i][j][k];
    for (u32 j = 0; j < ST.nint[rs]; ++j)
      for (u32 k = 0; k < 2; ++k) *iedges++ = ST.iedge[rs][i][j][k];
  }
  return 1;
}

/* ---- size-field producers ------------------------------------------------ */

/* dot_product (algebra.hpp) over n components */
static double dot_n(double const* a, double const* b, u32 n)
{
  double d = 0;
  for (u32 i = 0; i < n; ++i) d += a[i] * b[i];
  return d;
}

/* element_jacobian / invert_jacobian (jacobian.cpp:7-66) with
   invert_3x3 / invert_2x2 (algebra.hpp) */
static void or_invert_jacobian(u32 dim, double in[3][3], double out[3][3])
{
  if (dim == 3) {
    double tmp[3][3], c[3];
    cross3(in[0], in[1], c);
    double d = dot3(in[2], c);
    cross3(in[1], in[2], tmp[0]);
    cross3(in[2], in[0], tmp[1]);
    cross3(in[0], in[1], tmp[2]);
    double s = 1.0 / d;
    for (u32 i = 0; i < 3; ++i)
      for (u32 j = 0; j < 3; ++j) tmp[i][j] = tmp[i][j] * s;
    for (u32 i = 0; i < 3; ++i)
      for (u32 j = 0; j < 3; ++j) out[i][j] = tmp[j][i];
  } else if (dim == 2) {
    double nrm[2][2];
    for (u32 i = 0; i < 2; ++i)
      for (u32 j = 0; j < 2; ++j) {
        nrm[i][j] = 0;
        for (u32 k = 0; k < 3; ++k) nrm[i][j] += in[i][k] * in[j][k];
      }
    double d = nrm[0][0] * nrm[1][1] - nrm[0][1] * nrm[1][0];
    double inv[2][2];
    inv[0][0] = nrm[1][1] / d;
    inv[0][1] = -nrm[0][1] / d;
    inv[1][0] = -nrm[1][0] / d;
    inv[1][1] = nrm[0][0] / d;
    for (u32 i = 0; i < 3; ++i)
      for (u32 j = 0; j < 3; ++j) out[i][j] = 0;
    for (u32 i = 0; i < 3; ++i)
      for (u32 j = 0; j < 2; ++j)
        for (u32 k = 0; k < 2; ++k) out[i][j] += in[k][i] * inv[k][j];
  } else {
    double msq = dot3(in[0], in[0]);
    for (u32 i = 0; i < 3; ++i) out[i][0] = in[0][i] / msq;
    for (u32 i = 0; i < 3; ++i)
      for (u32 j = 1; j < 3; ++j) out[i][j] = 0;
  }
}

/* mesh_element_gradients (element_gradients.cpp:15-91) */
EXPORT void or_element_gradients(omesh* m, char const* name)
{
  u32 dim = m->dim, ne = count(m, dim), vpe = DEG[dim][0];
  otag* t = tags_find(&m->tags[0], name);
  if (!t) return;
  u32 nc = t->ncomps;
  double const* f = (double const*)t->data;
  u32 const* voe = ask_down(m, dim, 0);
  double const* x = coords_of(m);
  double* out = NEW(double, (size_t)ne * nc * 3);
  for (u32 i = 0; i < ne; ++i) {
    u32 const* ve = voe + (size_t)i * vpe;
    double ex[4][3];
    gather_x(x, ve, vpe, ex);
    double jac[3][3];
    for (u32 a = 0; a < 3; ++a)
      for (u32 b = 0; b < 3; ++b) jac[a][b] = 0;
    for (u32 a = 0; a < dim; ++a)
      for (u32 b = 0; b < 3; ++b) jac[b][a] = ex[a + 1][b] - ex[0][b];
    double jaci[3][3];
    or_invert_jacobian(dim, jac, jaci);
    double* g = out + (size_t)i * nc * 3;
    for (u32 k = 0; k < nc * 3; ++k) g[k] = 0;
    for (u32 j = 0; j < dim; ++j)
      for (u32 k = 0; k < nc; ++k)
        for (u32 l = 0; l < 3; ++l)
          g[k * 3 + l] += jaci[j][l] * (f[(size_t)ve[j + 1] * nc + k] - f[(size_t)ve[0] * nc + k]);
  }
  char gname[256];
  snprintf(gname, sizeof gname, "grad_%s", name);
  tags_add(&m->tags[dim], T_F64, gname, nc * 3, X_NOT, out);
}

/* mesh_recover_by_volume (recover_by_volume.cpp:10-68) */
EXPORT void or_recover_by_volume(omesh* m, char const* name)
{
  u32 dim = m->dim, nv = count(m, 0);
  otag* t = tags_find(&m->tags[dim], name);
  if (!t) return;
  u32 nc = t->ncomps;
  double const* f = (double const*)t->data;
  oup* u = ask_up(m, 0, dim);
  double* sizes = element_sizes(m);
  double* out = NEW(double, (size_t)nv * nc);
  for (u32 i = 0; i < nv; ++i) {
    double* o = out + (size_t)i * nc;
    for (u32 k = 0; k < nc; ++k) o[k] = 0;
    double size_sum = 0;
    for (u32 j = u->offs[i]; j < u->offs[i + 1]; ++j) {
      u32 e = u->adj[j];
      double es = sizes[e];
      size_sum += es;
      for (u32 k = 0; k < nc; ++k) o[k] += es * f[(size_t)e * nc + k];
    }
    for (u32 k = 0; k < nc; ++k) o[k] /= size_sum;
  }
  free(sizes);
  tags_add(&m->tags[0], T_F64, name, nc, X_NOT, out);
}

/* mesh_size_from_hessian (size_from_hessian.cpp:12-72) */
EXPORT void or_size_from_hessian(omesh* m, char const* hess_name, double const* weights,
    double min_h, double max_h)
{
  u32 nv = count(m, 0);
  otag* t = tags_find(&m->tags[0], hess_name);
  if (!t) return;
  u32 nhc = t->ncomps, nsol = nhc / 9;
  double const* hess = (double const*)t->data;
  double* out = NEW(double, nv);
  for (u32 i = 0; i < nv; ++i) {
    double const* hs = hess + (size_t)i * nhc;
    double total = 0;
    for (u32 j = 0; j < nsol; ++j) {
      double norm = sqrt(dot_n(hs, hs, 9));
      double hw = weights ? weights[j] : 1.0;
      total += hw * norm;
      hs += 9;
    }
    double o = max_h - total;
    if (o < min_h) o = min_h;
    out[i] = o;
  }
  tags_add(&m->tags[0], T_F64, "adapt_size", 1, X_NOT, out);
}

/* mesh_warp_to_limit (warp_to_limit.cpp:14-81); gives up (returns 2) after
   the halvings that leave the warp without effect, where the reference
   would loop forever */
EXPORT u32 or_warp_to_limit(omesh* m, double qual_floor)
{
  u32 n = count(m, 0) * 3;
  otag* xt = tags_find(&m->tags[0], "coordinates");
  otag* wt = tags_find(&m->tags[0], "warp");
  if (!xt || !wt) return 2;
  double const* x = (double const*)xt->data;
  double const* w = (double const*)wt->data;
  double* xo = NEW(double, n);
  double factor = 1;
  u32 hit = 0;
  for (u32 i = 0; i < n; ++i) xo[i] = factor * w[i] + x[i];
  u32 it = 0;
  for (;;) {
    /* exceeds_limit: min element quality of the warped coordinates */
    u32 dim = m->dim, ne = count(m, dim), vpe = DEG[dim][0];
    u32 const* voe = ask_down(m, dim, 0);
    double mq = DBL_MAX;
    for (u32 e = 0; e < ne; ++e) {
      double ex[4][3];
      gather_x(xo, voe + (size_t)e * vpe, vpe, ex);
      double q = element_quality(dim, ex);
      if (q < mq) mq = q;
    }
    if (!(mq < qual_floor)) break;
    if (++it > 1100) {
      free(xo);
      return 2;
    }
    hit = 1;
    factor /= 2;
    for (u32 i = 0; i < n; ++i) xo[i] = factor * w[i] + x[i];
  }
  double* wo = NEW(double, n);
  for (u32 i = 0; i < n; ++i) wo[i] = -factor * w[i] + w[i];
  tags_remove(&m->tags[0], "coordinates");
  tags_remove(&m->tags[0], "warp");
  tags_add(&m->tags[0], T_F64, "coordinates", 3, X_NOT, xo);
  tags_add(&m->tags[0], T_F64, "warp", 3, X_NOT, wo);
  return hit ? 0 : 1;
}
