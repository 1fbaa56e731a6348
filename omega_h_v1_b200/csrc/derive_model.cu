// Geometric classification of a mesh (mesh_derive_model, derive_model.cpp:
// 218-448): class_dim from boundary sides, crease angles and corners, then
// class_id from connected components of equal-order entities (bfs.cpp) and
// projection onto lower dimensions.
//
// This is one-time input preparation, done on the host from adjacency the
// device derived: the crease test calls acos, and running it on the host
// keeps every crease decision identical to the reference's.
#include <cmath>
#include <vector>

#include "mesh.hpp"

namespace osh {

template <class T>
static std::vector<T> to_host(T const* d, size_t n, cudaStream_t s)
{
  std::vector<T> h(n);
  if (n) CK(cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  return h;
}

struct HostUp {
  std::vector<u32> offs, adj;
};

static HostUp host_up(Mesh& m, u32 low, u32 high)
{
  UpAdj const& u = m.ask_up(low, high);
  HostUp h;
  u32 n = m.count(low);
  h.offs = to_host(u.offs, (size_t)n + 1, m.s);
  stream_sync(m.s);
  h.adj = to_host(u.adj, h.offs[n], m.s);
  stream_sync(m.s);
  return h;
}

static u32* upload(std::vector<u32> const& h, cudaStream_t s)
{
  u32* d = dalloc<u32>(h.size(), s);
  if (!h.empty())
    CK(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(u32), cudaMemcpyHostToDevice, s));
  stream_sync(s);
  return d;
}

void Mesh::derive_model(double crease)
{
  u32 const D = dim;
  if (D < 2) throw Failure(E_ARG, "classification needs a 2D or 3D mesh");
  u32 nel = count(D);
  std::vector<u32> ecd(nel, D);
  add_tag(D, T_U32, "class_dim", 1, X_NOT, upload(ecd, s));
  u32 ns = count(D - 1);
  HostUp es = host_up(*this, D - 1, D);
  std::vector<u32> bside(ns), scd(ns);
  for (u32 i = 0; i < ns; ++i) {
    bside[i] = (es.offs[i + 1] - es.offs[i]) < 2;
    scd[i] = D - bside[i];
  }
  add_tag(D - 1, T_U32, "class_dim", 1, X_NOT, upload(scd, s));
  std::vector<double> x = to_host(coords(), (size_t)count(0) * 3, s);
  u32 vps = deg(D - 1, 0);
  std::vector<u32> vos = to_host(ask_down(D - 1, 0), (size_t)ns * vps, s);
  stream_sync(s);
  // boundary side normals (derive_model.cpp:17-76)
  std::vector<double> nrm((size_t)ns * 3, 0.0);
  for (u32 i = 0; i < ns; ++i) {
    if (!bside[i]) continue;
    double* nn = &nrm[(size_t)i * 3];
    if (D - 1 == 1) {
      sub3(&x[vos[i * 2 + 1] * 3], &x[vos[i * 2] * 3], nn);
    } else {
      double b0[3], b1[3];
      sub3(&x[vos[i * 3 + 1] * 3], &x[vos[i * 3] * 3], b0);
      sub3(&x[vos[i * 3 + 2] * 3], &x[vos[i * 3] * 3], b1);
      cross3(b0, b1, nn);
    }
    double sc = 1.0 / std::sqrt(dot3(nn, nn));
    for (u32 k = 0; k < 3; ++k) nn[k] = nn[k] * sc;
  }
  // hinges: boundary marks, angles, creases (derive_model.cpp:78-138)
  u32 nh = count(D - 2);
  HostUp sh = host_up(*this, D - 2, D - 1);
  std::vector<u32> bh(nh, 0), crease_h(nh, 0), hcd(nh);
  for (u32 i = 0; i < nh; ++i) {
    for (u32 j = sh.offs[i]; j < sh.offs[i + 1]; ++j)
      if (bside[sh.adj[j]]) {
        bh[i] = 1;
        break;
      }
    double ang = 0;
    if (bh[i]) {
      u32 adj[2] = {0, 0}, na = 0;
      for (u32 j = sh.offs[i]; j < sh.offs[i + 1]; ++j)
        if (bside[sh.adj[j]] && na < 2) adj[na++] = sh.adj[j];
      ang = std::acos(dot3(&nrm[adj[0] * 3], &nrm[adj[1] * 3]));
    }
    crease_h[i] = ang > crease;
    hcd[i] = D - bh[i] - crease_h[i];
  }
  add_tag(D - 2, T_U32, "class_dim", 1, X_NOT, upload(hcd, s));
  if (D == 3) {
    // corners and vertex class_dim (derive_model.cpp:140-216)
    u32 nv = count(0);
    HostUp ev = host_up(*this, 0, 1);
    std::vector<u32> vcd(nv);
    for (u32 i = 0; i < nv; ++i) {
      u32 nin = 0, d = 3;
      for (u32 j = ev.offs[i]; j < ev.offs[i + 1]; ++j) {
        u32 e = ev.adj[j];
        if (crease_h[e]) ++nin;
        if (hcd[e] < d) d = hcd[e];
      }
      vcd[i] = d - (nin > 2 ? 1u : 0u);
    }
    add_tag(0, T_U32, "class_dim", 1, X_NOT, upload(vcd, s));
  }
  // class ids (derive_model.cpp:414-442)
  std::vector<std::vector<u32>> cd(D + 1), cid(D + 1);
  for (u32 d = 0; d <= D; ++d) {
    cd[d] = to_host(static_cast<u32 const*>(find_tag(d, "class_dim")->data), count(d), s);
  }
  stream_sync(s);
  {
    u32 nv = count(0), k = 0;
    cid[0].assign(nv, INV);
    for (u32 i = 0; i < nv; ++i)
      if (cd[0][i] == 0) cid[0][i] = k++;
  }
  for (u32 d = 1; d <= D; ++d) {
    // components of entities classified on d, joined through sides also
    // classified on d, numbered by their smallest member
    u32 n = count(d), spd = deg(d, d - 1);
    std::vector<u32> sod = to_host(ask_down(d, d - 1), (size_t)n * spd, s);
    stream_sync(s);
    HostUp dos = host_up(*this, d - 1, d);
    std::vector<u32>& id = cid[d];
    id.assign(n, INV);
    std::vector<u32> queue(n);
    u32 comp = 0;
    for (u32 i = 0; i < n; ++i) {
      if (cd[d][i] != d || id[i] != INV) continue;
      u32 b = 0, e = 0;
      queue[e++] = i;
      id[i] = comp;
      while (b != e) {
        u32 u = queue[b++];
        for (u32 j = 0; j < spd; ++j) {
          u32 sd = sod[(size_t)u * spd + j];
          if (cd[d - 1][sd] != d) continue;
          for (u32 l = dos.offs[sd]; l < dos.offs[sd + 1]; ++l) {
            u32 o = dos.adj[l];
            if (o == u || cd[d][o] != d) continue;
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
  }
  for (u32 dd = 1; dd <= D; ++dd) {
    // project_class_id_onto (derive_model.cpp:392-412)
    u32 d = D - dd, nl = count(d);
    HostUp u = host_up(*this, d, d + 1);
    for (u32 i = 0; i < nl; ++i)
      for (u32 j = u.offs[i]; j < u.offs[i + 1]; ++j)
        if (cd[d + 1][u.adj[j]] == cd[d][i]) cid[d][i] = cid[d + 1][u.adj[j]];
  }
  for (u32 d = 0; d <= D; ++d) add_tag(d, T_U32, "class_id", 1, X_NOT, upload(cid[d], s));
  // the reference adds tags in this order: dim, dim-1, ..., then class_id 0..dim
  full = true;
}

}  // namespace osh
