// Geometric classification of a mesh on the device (mesh_derive_model,
// derive_model.cpp:218-448): class_dim from boundary sides, crease angles and
// corners, then class_id from connected components of equally classified
// entities (the reference's breadth-first search, bfs.cpp) and projection
// onto lower dimensions.
//
// Crease test: the reference compares acos(n0 . n1) with the crease angle.
// acos is decreasing, so every hinge whose dot product lies more than 1e-9
// away from cos(crease) is decided on the device by comparing the dot
// product; the few inside that band are sent to the host, which applies the
// reference's own test with std::acos, so every decision is the reference's.
//
// Components: union-find in which a root only ever hooks under a smaller
// root, so the final root of a component is its smallest member, and the
// components are numbered in the order of their smallest members, which is
// the order in which the reference's search meets them.
#include <cmath>
#include <vector>

#include "mesh.hpp"

namespace osh {

namespace {

constexpr u32 UF_CAP = 1u << 24;  // bound on any union-find walk or retry loop

// boundary sides (fewer than two elements) and their class_dim
__global__ void k_side_class(u32 ns, u32 D, u32 const* __restrict__ offs,
    u32* __restrict__ bside, u32* __restrict__ scd)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  u32 b = (offs[i + 1] - offs[i]) < 2 ? 1u : 0u;
  bside[i] = b;
  scd[i] = D - b;
}

// unit normals of boundary sides (derive_model.cpp:17-76): the edge vector
// in 2D, the triangle's (v1 - v0) x (v2 - v0) in 3D
__global__ void k_side_normals(u32 ns, u32 D, u32 const* __restrict__ vos,
    double const* __restrict__ x, u32 const* __restrict__ bside, double* __restrict__ nrm)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  double nn[3] = {0.0, 0.0, 0.0};
  if (bside[i]) {
    if (D == 2) {
      double a[3], b[3];
      load3(x, vos[i * 2 + 1], a);
      load3(x, vos[i * 2], b);
      sub3(a, b, nn);
    } else {
      double p0[3], p1[3], p2[3], b0[3], b1[3];
      load3(x, vos[i * 3], p0);
      load3(x, vos[i * 3 + 1], p1);
      load3(x, vos[i * 3 + 2], p2);
      sub3(p1, p0, b0);
      sub3(p2, p0, b1);
      cross3(b0, b1, nn);
    }
    double sc = 1.0 / sqrt(dot3(nn, nn));
    for (u32 k = 0; k < 3; ++k) nn[k] = nn[k] * sc;
  }
  nrm[i * 3 + 0] = nn[0];
  nrm[i * 3 + 1] = nn[1];
  nrm[i * 3 + 2] = nn[2];
}

// hinges (derive_model.cpp:78-138): on the boundary if any adjacent side is;
// the crease angle is between the first two boundary sides in row order (a
// missing second side reads side 0, as the reference's zeroed pair does)
__global__ void k_hinge_class(u32 nh, u32 const* __restrict__ offs, u32 const* __restrict__ adj,
    u32 const* __restrict__ bside, double const* __restrict__ nrm, double cos_lo,
    double cos_hi, u32* __restrict__ bh, u32* __restrict__ crease, double* __restrict__ dots,
    u32* __restrict__ namb, u32* __restrict__ amb)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nh) return;
  u32 a[2] = {0, 0}, na = 0;
  for (u32 j = offs[i]; j < offs[i + 1]; ++j)
    if (bside[adj[j]] && na < 2) a[na++] = adj[j];
  u32 b = na > 0 ? 1u : 0u, c = 0;
  if (b) {
    double d = dot3(nrm + (size_t)a[0] * 3, nrm + (size_t)a[1] * 3);
    dots[i] = d;
    if (d < cos_lo) {
      c = 1;
    } else if (!(d > cos_hi)) {
      // within the band, or NaN: the host decides with acos
      u32 k = atomicAdd(namb, 1u);
      amb[k] = i;
    }
  }
  bh[i] = b;
  crease[i] = c;
}

__global__ void k_set_flags(u32 n, u32 const* __restrict__ idx, u32 const* __restrict__ val,
    u32* __restrict__ out)
{
  pdl_wait();
  u32 k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[idx[k]] = val[k];
}

__global__ void k_hinge_cd(u32 nh, u32 D, u32 const* __restrict__ bh,
    u32 const* __restrict__ crease, u32* __restrict__ hcd)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nh) hcd[i] = D - bh[i] - crease[i];
}

// 3D vertices (derive_model.cpp:140-216): the lowest class_dim of their
// edges, one lower again at a corner of more than two crease edges
__global__ void k_vertex_class(u32 nv, u32 const* __restrict__ offs, u32 const* __restrict__ adj,
    u32 const* __restrict__ crease, u32 const* __restrict__ hcd, u32* __restrict__ vcd)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  u32 nin = 0, d = 3;
  for (u32 j = offs[i]; j < offs[i + 1]; ++j) {
    u32 e = adj[j];
    if (crease[e]) ++nin;
    if (hcd[e] < d) d = hcd[e];
  }
  vcd[i] = d - (nin > 2 ? 1u : 0u);
}

__global__ void k_is_value(u32 n, u32 const* __restrict__ a, u32 v, u32* __restrict__ out)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] == v ? 1u : 0u;
}

__global__ void k_vertex_ids(u32 n, u32 const* __restrict__ cd, u32 const* __restrict__ scan,
    u32* __restrict__ cid)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) cid[i] = cd[i] == 0 ? scan[i] : INV;
}

__device__ u32 uf_find(u32* parent, u32 x, u32* fail)
{
  for (u32 it = 0; it < UF_CAP; ++it) {
    u32 p = __ldcg(parent + x);
    if (p == x) return x;
    u32 gp = __ldcg(parent + p);
    if (gp != p) atomicMin(parent + x, gp);  // path halving; parents only shrink
    x = gp;
  }
  atomicOr(fail, 1u);
  return x;
}

__global__ void k_cc_init(u32 n, u32 const* __restrict__ cd, u32 d, u32* __restrict__ parent)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) parent[i] = cd[i] == d ? i : INV;
}

// entity u and every other entity classified on d that shares with it a
// side classified on d are in one component
__global__ void k_cc_hook(u32 n, u32 spd, u32 const* __restrict__ sod,
    u32 const* __restrict__ cds, u32 const* __restrict__ offs, u32 const* __restrict__ adj,
    u32 const* __restrict__ cdd, u32 d, u32* parent, u32* fail)
{
  pdl_wait();
  u32 t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * spd) return;
  u32 u = t / spd;
  if (cdd[u] != d) return;
  u32 sd = sod[t];
  if (cds[sd] != d) return;
  for (u32 j = offs[sd]; j < offs[sd + 1]; ++j) {
    u32 o = adj[j];
    if (o == u || cdd[o] != d) continue;
    u32 ra = uf_find(parent, u, fail), rb = uf_find(parent, o, fail);
    u32 it = 0;
    while (ra != rb) {
      if (++it > UF_CAP) {
        atomicOr(fail, 1u);
        break;
      }
      if (ra < rb) {
        u32 x = ra;
        ra = rb;
        rb = x;
      }
      u32 old = atomicCAS(parent + ra, ra, rb);
      if (old == ra) break;
      ra = uf_find(parent, old, fail);
      rb = uf_find(parent, rb, fail);
    }
  }
}

__global__ void k_cc_flatten(u32 n, u32* parent, u32* __restrict__ is_root, u32* fail)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 p = parent[i];
  if (p == INV) {
    is_root[i] = 0;
    return;
  }
  u32 r = uf_find(parent, i, fail);
  parent[i] = r;
  is_root[i] = r == i ? 1u : 0u;
}

__global__ void k_cc_ids(u32 n, u32 const* __restrict__ parent, u32 const* __restrict__ scan,
    u32* __restrict__ cid)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 p = parent[i];
  cid[i] = p == INV ? INV : scan[p];
}

// project_class_id_onto (derive_model.cpp:392-412): the last upward entity
// (row order) with the same class_dim gives its class_id
__global__ void k_project_ids(u32 n, u32 const* __restrict__ offs, u32 const* __restrict__ adj,
    u32 const* __restrict__ cd_hi, u32 const* __restrict__ cid_hi,
    u32 const* __restrict__ cd_lo, u32* __restrict__ cid_lo)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 c = cd_lo[i], id = cid_lo[i];
  for (u32 j = offs[i]; j < offs[i + 1]; ++j)
    if (cd_hi[adj[j]] == c) id = cid_hi[adj[j]];
  cid_lo[i] = id;
}

}  // namespace

void Mesh::derive_model(double crease_angle)
{
  u32 const D = dim;
  if (D < 2) throw Failure(E_ARG, "classification needs a 2D or 3D mesh");
  u32 nel = count(D);
  u32* cd[4] = {nullptr, nullptr, nullptr, nullptr};
  // elements
  cd[D] = dalloc<u32>(nel, s);
  fill_u32(cd[D], nel, D, s);
  add_tag(D, T_U32, "class_dim", 1, X_NOT, cd[D]);
  // sides
  u32 ns = count(D - 1);
  UpAdj const& es = ask_up(D - 1, D, false);
  u32* bside = dalloc<u32>(ns, s);
  cd[D - 1] = dalloc<u32>(ns, s);
  if (ns) {
    CK(launch_kernel(k_side_class, dim3(grid_for(ns)), dim3(BLOCK), 0, s, ns, D, es.offs, bside, cd[D - 1]));
    CK_LAUNCH();
  }
  add_tag(D - 1, T_U32, "class_dim", 1, X_NOT, cd[D - 1]);
  double* nrm = dalloc<double>((size_t)ns * 3, s);
  if (ns) {
    CK(launch_kernel(k_side_normals, dim3(grid_for(ns)), dim3(BLOCK), 0, s, ns, D, ask_down(D - 1, 0), coords(), bside,
        nrm));
    CK_LAUNCH();
  }
  // hinges
  u32 nh = count(D - 2);
  UpAdj const& sh = ask_up(D - 2, D - 1, true);
  u32* bh = dalloc<u32>(nh, s);
  u32* crease = dalloc<u32>(nh, s);
  double* dots = dalloc<double>(nh, s);
  u32* amb = dalloc<u32>(nh ? nh : 1, s);
  u32* namb = mb->dev + 24;
  CK(cudaMemsetAsync(namb, 0, sizeof(u32), s));
  double cc = std::cos(crease_angle);
  if (nh) {
    CK(launch_kernel(k_hinge_class, dim3(grid_for(nh)), dim3(BLOCK), 0, s, nh, sh.offs, sh.adj, bside, nrm, cc - 1e-9,
        cc + 1e-9, bh, crease, dots, namb, amb));
    CK_LAUNCH();
  }
  mb->fetch(s, 25);
  u32 na = mb->host[24];
  if (na) {
    // the reference's own test for the hinges inside the band
    std::vector<u32> idx(na), val(na);
    std::vector<double> dv(na);
    CK(cudaMemcpyAsync(idx.data(), amb, sizeof(u32) * na, cudaMemcpyDeviceToHost, s));
    stream_sync(s);
    double* dsel = dalloc<double>(na, s);
    for (u32 k = 0; k < na; ++k)
      CK(cudaMemcpyAsync(dsel + k, dots + idx[k], sizeof(double), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(dv.data(), dsel, sizeof(double) * na, cudaMemcpyDeviceToHost, s));
    stream_sync(s);
    dev_free(dsel, s);
    for (u32 k = 0; k < na; ++k) val[k] = std::acos(dv[k]) > crease_angle ? 1u : 0u;
    u32* di = dalloc<u32>(2 * (size_t)na, s);
    CK(cudaMemcpyAsync(di, idx.data(), sizeof(u32) * na, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(di + na, val.data(), sizeof(u32) * na, cudaMemcpyHostToDevice, s));
    CK(launch_kernel(k_set_flags, dim3(grid_for(na)), dim3(BLOCK), 0, s, na, di, di + na, crease));
    CK_LAUNCH();
    stream_sync(s);
    dev_free(di, s);
  }
  dev_free(dots, s);
  dev_free(amb, s);
  dev_free(nrm, s);
  cd[D - 2] = dalloc<u32>(nh, s);
  if (nh) {
    CK(launch_kernel(k_hinge_cd, dim3(grid_for(nh)), dim3(BLOCK), 0, s, nh, D, bh, crease, cd[D - 2]));
    CK_LAUNCH();
  }
  add_tag(D - 2, T_U32, "class_dim", 1, X_NOT, cd[D - 2]);
  if (D == 3) {
    u32 nv = count(0);
    UpAdj const& ev = ask_up(0, 1, false);
    cd[0] = dalloc<u32>(nv, s);
    if (nv) {
      CK(launch_kernel(k_vertex_class, dim3(grid_for(nv)), dim3(BLOCK), 0, s, nv, ev.offs, ev.adj, crease, cd[D - 2],
          cd[0]));
      CK_LAUNCH();
    }
    add_tag(0, T_U32, "class_dim", 1, X_NOT, cd[0]);
  }
  dev_free(bside, s);
  dev_free(bh, s);
  dev_free(crease, s);
  // class ids (derive_model.cpp:414-442)
  u32* cid[4] = {nullptr, nullptr, nullptr, nullptr};
  {
    u32 nv = count(0);
    u32* f = dalloc<u32>(nv ? nv : 1, s);
    if (nv) {
      CK(launch_kernel(k_is_value, dim3(grid_for(nv)), dim3(BLOCK), 0, s, nv, cd[0], 0, f));
      CK_LAUNCH();
    }
    u32* sc = exscan_new(f, nv, s);
    cid[0] = dalloc<u32>(nv, s);
    if (nv) {
      CK(launch_kernel(k_vertex_ids, dim3(grid_for(nv)), dim3(BLOCK), 0, s, nv, cd[0], sc, cid[0]));
      CK_LAUNCH();
    }
    dev_free(sc, s);
    dev_free(f, s);
  }
  u32* fail = mb->dev + 25;
  CK(cudaMemsetAsync(fail, 0, sizeof(u32), s));
  for (u32 d = 1; d <= D; ++d) {
    u32 n = count(d), spd = deg(d, d - 1);
    u32 const* sod = ask_down(d, d - 1);
    UpAdj const& dos = ask_up(d - 1, d, false);
    cid[d] = dalloc<u32>(n, s);
    u32* roots = dalloc<u32>(n ? n : 1, s);
    if (n) {
      CK(launch_kernel(k_cc_init, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, cd[d], d, cid[d]));
      CK_LAUNCH();
      CK(launch_kernel(k_cc_hook, dim3(grid_for((u64)n * spd)), dim3(BLOCK), 0, s, n, spd, sod, cd[d - 1], dos.offs,
          dos.adj, cd[d], d, cid[d], fail));
      CK_LAUNCH();
      CK(launch_kernel(k_cc_flatten, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, cid[d], roots, fail));
      CK_LAUNCH();
    }
    u32* sc = exscan_new(roots, n, s);
    if (n) {
      CK(launch_kernel(k_cc_ids, dim3(grid_for(n)), dim3(BLOCK), 0, s, n, cid[d], sc, cid[d]));
      CK_LAUNCH();
    }
    dev_free(sc, s);
    dev_free(roots, s);
  }
  mb->fetch(s, 26);
  if (mb->host[25]) {
    for (u32 d = 0; d <= D; ++d) dev_free(cid[d], s);
    throw Failure(E_TIMEOUT, "classification: a union-find walk exceeded its bound");
  }
  for (u32 dd = 1; dd <= D; ++dd) {
    u32 d = D - dd, nl = count(d);
    UpAdj const& u = ask_up(d, d + 1, true);
    if (nl) {
      CK(launch_kernel(k_project_ids, dim3(grid_for(nl)), dim3(BLOCK), 0, s, nl, u.offs, u.adj, cd[d + 1], cid[d + 1],
          cd[d], cid[d]));
      CK_LAUNCH();
    }
  }
  for (u32 d = 0; d <= D; ++d) add_tag(d, T_U32, "class_id", 1, X_NOT, cid[d]);
  // the reference adds tags in this order: class_dim of dim, dim-1, ...,
  // then class_id of 0..dim
  full = true;
}

}  // namespace osh
