// VTU mesh files: the reference's reader and writer (vtk_io.cpp) with the
// same file layout byte for byte, so that files move between the two
// libraries and the reference's own golden-file diffs hold.
//
// File layout (vtk_io.cpp:466-517): a VTKFile/UnstructuredGrid with one
// Piece carrying NumberOfPoints/Cells (+ NumberOfEdges/Faces when the mesh
// holds them) and Rep="Full"|"Reduced"; Points (the "coordinates" tag),
// Edges, Faces and Cells connectivity (+ offsets and types), then
// PointData / EdgeData / FaceData / CellData with every tag in list order.
// Binary arrays are base64 of a UInt32 byte count followed by base64 of the
// raw little-endian values (two separately padded strings,
// vtk_io.cpp:149-171); with zlib, a {1, size, size, compressed size} header
// and one zlib block. ASCII arrays print one entity per line.
//
// Work split: base64 encoding and decoding of uncompressed arrays run on the
// device (one thread per 3-byte / 4-character unit; the whole file is
// copied to the device once for reading); ASCII formatting, zlib and the
// markup stay on the host, where the reference's printf / scanf
// conversions fix the bytes.
#include <zlib.h>

#include <cerrno>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "mesh.hpp"
#include "vtk_io.hpp"

namespace osh {

namespace {

char const* const TYPE_NAMES[4] = {"UInt8", "UInt32", "UInt64", "Float64"};
// simplex_types (vtk_io.cpp:39-44): VTK_VERTEX, VTK_LINE, VTK_TRIANGLE, VTK_TETRA
unsigned char const CELL_TYPES[4] = {1, 3, 5, 10};

[[noreturn]] void io_fail(std::string const& what)
{
  throw Failure(E_IO, what);
}

// ---------------------------------------------------------------------------
// base64, RFC 4648 alphabet, '=' padding (base64.cpp)

__host__ __device__ inline char b64_char(u32 v)
{
  return v < 26 ? char('A' + v) : v < 52 ? char('a' + v - 26) : v < 62 ? char('0' + v - 52)
                                                                       : v == 62 ? '+' : '/';
}

// value of a base64 character; '=' reads as 0 (base64.cpp:49); 64 = not base64
__host__ __device__ inline u32 b64_value(u32 c)
{
  if (c >= 'A' && c <= 'Z') return c - 'A';
  if (c >= 'a' && c <= 'z') return c - 'a' + 26;
  if (c >= '0' && c <= '9') return c - '0' + 52;
  if (c == '+') return 62;
  if (c == '/') return 63;
  if (c == '=') return 0;
  return 64;
}

// unit u: bytes [3u, 3u+3) of `in` -> characters [4u, 4u+4) of `out`
__global__ void k_b64_encode(unsigned char const* __restrict__ in, u64 nbytes,
    char4* __restrict__ out)
{
  pdl_wait();
  u64 u = blockIdx.x * (u64)blockDim.x + threadIdx.x;
  u64 b = u * 3;
  if (b >= nbytes) return;
  u32 rem = nbytes - b < 3 ? u32(nbytes - b) : 3u;
  u32 b0 = in[b];
  u32 b1 = rem > 1 ? in[b + 1] : 0u;
  u32 b2 = rem > 2 ? in[b + 2] : 0u;
  char4 o;
  o.x = b64_char(b0 >> 2);
  o.y = b64_char(((b0 << 4) & 0x30u) | (b1 >> 4));
  o.z = rem > 1 ? b64_char(((b1 << 2) & 0x3cu) | (b2 >> 6)) : '=';
  o.w = rem > 2 ? b64_char(b2 & 0x3fu) : '=';
  out[u] = o;
}

// unit u: characters [4u, 4u+4) of `in` -> bytes [3u, 3u+3) of `out`, cut at
// nbytes; a character outside the alphabet sets *bad
__global__ void k_b64_decode(char const* __restrict__ in, u64 nbytes,
    unsigned char* __restrict__ out, u32* bad)
{
  pdl_wait();
  u64 u = blockIdx.x * (u64)blockDim.x + threadIdx.x;
  u64 b = u * 3;
  if (b >= nbytes) return;
  u32 v[4];
  u32 ok = 1;
  for (u32 k = 0; k < 4; ++k) {
    v[k] = b64_value((unsigned char)in[u * 4 + k]);
    if (v[k] > 63) {
      ok = 0;
      v[k] = 0;
    }
  }
  if (!ok) atomicOr(bad, 1u);
  out[b] = (unsigned char)(((v[0] << 2) & 0xfcu) | ((v[1] >> 4) & 0x03u));
  if (b + 1 < nbytes) out[b + 1] = (unsigned char)(((v[1] << 4) & 0xf0u) | ((v[2] >> 2) & 0x0fu));
  if (b + 2 < nbytes) out[b + 2] = (unsigned char)(((v[2] << 6) & 0xc0u) | (v[3] & 0x3fu));
}

// reverse the bytes of every `width`-byte value (generic_swap_if_needed)
__global__ void k_swap_bytes(unsigned char* a, u64 n, u32 width)
{
  pdl_wait();
  u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned char* p = a + i * width;
  for (u32 j = 0; j < width / 2; ++j) {
    unsigned char t = p[j];
    p[j] = p[width - 1 - j];
    p[width - 1 - j] = t;
  }
}

// offsets (k + 1) * vpe and the element type code, for the Cells arrays
__global__ void k_cell_arrays(u32 n, u32 vpe, u32* __restrict__ offs, unsigned char* types,
    unsigned char type)
{
  pdl_wait();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  offs[i] = (i + 1) * vpe;
  types[i] = type;
}

u32 encode_grid(u64 nbytes)
{
  u64 units = (nbytes + 2) / 3;
  return (u32)((units + BLOCK - 1) / BLOCK);
}

std::string b64_host(void const* data, size_t n)
{
  unsigned char const* in = static_cast<unsigned char const*>(data);
  std::string out;
  out.resize((n + 2) / 3 * 4);
  for (size_t b = 0, u = 0; b < n; b += 3, ++u) {
    size_t rem = n - b < 3 ? n - b : 3;
    u32 b0 = in[b], b1 = rem > 1 ? in[b + 1] : 0u, b2 = rem > 2 ? in[b + 2] : 0u;
    out[u * 4 + 0] = b64_char(b0 >> 2);
    out[u * 4 + 1] = b64_char(((b0 << 4) & 0x30u) | (b1 >> 4));
    out[u * 4 + 2] = rem > 1 ? b64_char(((b1 << 2) & 0x3cu) | (b2 >> 6)) : '=';
    out[u * 4 + 3] = rem > 2 ? b64_char(b2 & 0x3fu) : '=';
  }
  return out;
}

// decode nbytes from the characters at s (at least 4 ceil(nbytes / 3) of them)
void b64_host_decode(char const* s, size_t nbytes, unsigned char* out)
{
  for (size_t b = 0, u = 0; b < nbytes; b += 3, ++u) {
    u32 v[4];
    for (u32 k = 0; k < 4; ++k) {
      v[k] = b64_value((unsigned char)s[u * 4 + k]);
      if (v[k] > 63) io_fail("bad base64 character");
    }
    out[b] = (unsigned char)(((v[0] << 2) & 0xfcu) | ((v[1] >> 4) & 0x03u));
    if (b + 1 < nbytes) out[b + 1] = (unsigned char)(((v[1] << 4) & 0xf0u) | ((v[2] >> 2) & 0x0fu));
    if (b + 2 < nbytes) out[b + 2] = (unsigned char)(((v[2] << 6) & 0xc0u) | (v[3] & 0x3fu));
  }
}

size_t b64_chars(size_t nbytes) { return (nbytes + 2) / 3 * 4; }

bool host_little_endian()
{
  u32 one = 1;
  unsigned char c;
  std::memcpy(&c, &one, 1);
  return c == 1;
}

void swap_host(void* a, size_t n, u32 width)
{
  unsigned char* p = static_cast<unsigned char*>(a);
  for (size_t i = 0; i < n; ++i)
    for (u32 j = 0; j < width / 2; ++j) {
      unsigned char t = p[i * width + j];
      p[i * width + j] = p[i * width + width - 1 - j];
      p[i * width + width - 1 - j] = t;
    }
}

// ---------------------------------------------------------------------------
// markup: attribute lookup as the reference does it (vtk_io.cpp:65-82): the
// first occurrence of name=" in the line, value up to the next quote

bool try_attrib(std::string const& line, char const* name, std::string& val)
{
  std::string key = std::string(name) + "=\"";
  size_t p = line.find(key);
  if (p == std::string::npos) return false;
  size_t a = p + key.size();
  size_t e = line.find('"', a);
  if (e == std::string::npos || e == a) return false;
  val = line.substr(a, e - a);
  return true;
}

std::string attrib(std::string const& line, char const* name)
{
  std::string v;
  if (!try_attrib(line, name, v))
    io_fail(std::string("missing attribute ") + name + " in: " + line.substr(0, 200));
  return v;
}

bool try_int_attrib(std::string const& line, char const* name, u32* out)
{
  std::string v;
  if (!try_attrib(line, name, v)) return false;
  *out = (u32)atoi(v.c_str());
  return true;
}

struct ArrayHead {
  u32 type = T_U32;
  std::string name;
  u32 ncomps = 1;
  bool ascii = false;
};

ArrayHead parse_head(std::string const& line)
{
  ArrayHead h;
  std::string t = attrib(line, "type");
  u32 k = 0;
  for (; k < 4; ++k)
    if (t == TYPE_NAMES[k]) break;
  if (k == 4) io_fail("unsupported array type " + t);
  h.type = k;
  h.name = attrib(line, "Name");
  if (!try_int_attrib(line, "NumberOfComponents", &h.ncomps)) h.ncomps = 1;
  std::string f = attrib(line, "format");
  if (f == "ascii")
    h.ascii = true;
  else if (f != "binary")
    io_fail("unsupported array format " + f);
  return h;
}

// ---------------------------------------------------------------------------
// reading

struct Reader {
  cudaStream_t s;
  char* text = nullptr;   // the whole file, pinned host memory
  size_t size = 0;
  size_t pos = 0;
  char* dtext = nullptr;  // the same bytes on the device (first binary array)
  u32* dbad = nullptr;
  bool swap = false;      // file byte order differs from this host's
  bool compressed = false;

  Reader(char const* path, cudaStream_t st) : s(st)
  {
    FILE* f = fopen(path, "rb");
    if (!f) io_fail(std::string("cannot open ") + path + ": " + strerror(errno));
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (n < 0) {
      fclose(f);
      io_fail(std::string("cannot size ") + path);
    }
    size = (size_t)n;
    if (cudaMallocHost(&text, size + 1) != cudaSuccess) {
      fclose(f);
      throw Failure(E_NOMEM, "pinned buffer for a VTU file");
    }
    size_t got = fread(text, 1, size, f);
    fclose(f);
    if (got != size) io_fail(std::string("short read of ") + path);
    text[size] = '\0';
  }
  ~Reader()
  {
    if (dtext) {
      cudaStreamSynchronize(s);
      cudaFreeAsync(dtext, s);
      cudaFreeAsync(dbad, s);
    }
    if (text) cudaFreeHost(text);
  }

  bool next_line(std::string& line)
  {
    if (pos >= size) return false;
    char const* nl = static_cast<char const*>(memchr(text + pos, '\n', size - pos));
    size_t e = nl ? (size_t)(nl - text) : size;
    line.assign(text + pos, e - pos);
    pos = e < size ? e + 1 : e;
    return true;
  }
  // seek_prefix (files.cpp:104-112): the next line that starts with prefix
  void seek(char const* prefix, std::string& line)
  {
    size_t pl = strlen(prefix);
    while (next_line(line))
      if (line.compare(0, pl, prefix) == 0) return;
    io_fail(std::string("no ") + prefix + " in the file");
  }
  bool next_is(char const* prefix, std::string& line)
  {
    if (!next_line(line)) return false;
    return line.compare(0, strlen(prefix), prefix) == 0;
  }

  // the run of base64 characters at pos (base64_fread, base64.cpp:126-141)
  size_t b64_run()
  {
    size_t e = pos;
    while (e < size && b64_value((unsigned char)text[e]) < 64) ++e;
    return e - pos;
  }

  void to_device()
  {
    if (dtext) return;
    dtext = dalloc<char>(size + 1, s);
    dbad = dalloc<u32>(1, s);
    CK(cudaMemcpyAsync(dtext, text, size, cudaMemcpyHostToDevice, s));
  }

  // read_binary_array (vtk_io.cpp:184-218) into device memory
  void* binary(ArrayHead const& h, u64 nvals)
  {
    u32 esz = tag_esz(h.type);
    u64 nbytes = nvals * esz;
    size_t run = b64_run();
    void* out = dev_alloc(nbytes ? nbytes : 1, s);
    try {
      if (!compressed) {
        // a UInt32 byte count, then the values
        size_t head = b64_chars(4);
        if (run < head + b64_chars(nbytes)) io_fail("binary array " + h.name + " is short");
        if (nbytes) {
          to_device();
          CK(cudaMemsetAsync(dbad, 0, sizeof(u32), s));
          CK(launch_kernel(k_b64_decode, dim3(encode_grid(nbytes)), dim3(BLOCK), 0, s, dtext + pos + head, nbytes,
              static_cast<unsigned char*>(out), dbad));
          CK_LAUNCH();
          if (swap && esz > 1) {
            CK(launch_kernel(k_swap_bytes, dim3(grid_for(nvals)), dim3(BLOCK), 0, s, static_cast<unsigned char*>(out),
                nvals, esz));
            CK_LAUNCH();
          }
          u32 bad = 0;
          CK(cudaMemcpyAsync(&bad, dbad, sizeof(u32), cudaMemcpyDeviceToHost, s));
          stream_sync(s);
          if (bad) io_fail("bad base64 character in array " + h.name);
        }
      } else {
        // {nblocks, block size, last block size, compressed sizes...}: the
        // reference writes and reads exactly one block
        size_t head = b64_chars(16);
        if (run < head) io_fail("binary array " + h.name + " is short");
        u32 hdr[4];
        b64_host_decode(text + pos, 16, reinterpret_cast<unsigned char*>(hdr));
        if (swap) swap_host(hdr, 4, 4);
        if (hdr[0] != 1) io_fail("compressed array " + h.name + " has more than one block");
        size_t csize = hdr[3];
        if (run < head + b64_chars(csize)) io_fail("compressed array " + h.name + " is short");
        std::vector<unsigned char> comp(csize), raw(nbytes ? nbytes : 1);
        b64_host_decode(text + pos + head, csize, comp.data());
        uLongf got = nbytes;
        if (uncompress(raw.data(), &got, comp.data(), csize) != Z_OK || got != nbytes)
          io_fail("zlib cannot inflate array " + h.name);
        if (swap && esz > 1) swap_host(raw.data(), nvals, esz);
        CK(cudaMemcpyAsync(out, raw.data(), nbytes, cudaMemcpyHostToDevice, s));
        stream_sync(s);
      }
    } catch (...) {
      dev_free(out, s);
      throw;
    }
    pos += run;
    return out;
  }

  // read_ascii_array (vtk_io.cpp:265-309): scanf conversions of each value
  void* ascii(ArrayHead const& h, u64 nvals)
  {
    u32 esz = tag_esz(h.type);
    std::vector<unsigned char> host(nvals * esz ? nvals * esz : 1);
    char* p = text + pos;
    char* end_all = text + size;
    for (u64 i = 0; i < nvals; ++i) {
      char* e = nullptr;
      errno = 0;
      if (h.type == T_F64) {
        double v = strtod(p, &e);
        std::memcpy(&host[i * 8], &v, 8);
      } else {
        unsigned long v = strtoul(p, &e, 10);
        if (h.type == T_U8) {
          host[i] = (unsigned char)v;
        } else if (h.type == T_U32) {
          u32 w = (u32)v;
          std::memcpy(&host[i * 4], &w, 4);
        } else {
          std::memcpy(&host[i * 8], &v, 8);
        }
      }
      if (e == p || e > end_all) io_fail("ascii array " + h.name + " is short");
      p = e;
    }
    pos = (size_t)(p - text);
    void* out = dev_alloc(nvals * esz ? nvals * esz : 1, s);
    if (nvals) CK(cudaMemcpyAsync(out, host.data(), nvals * esz, cudaMemcpyHostToDevice, s));
    stream_sync(s);
    return out;
  }

  // read_array (vtk_io.cpp:382-400): the values that follow a DataArray line
  void* array(ArrayHead const& h, u64 nents)
  {
    u64 nvals = nents * h.ncomps;
    void* d = h.ascii ? ascii(h, nvals) : binary(h, nvals);
    std::string line;
    try {
      seek("</DataArray", line);
    } catch (...) {
      dev_free(d, s);
      throw;
    }
    return d;
  }
};

// read_tags (vtk_io.cpp:621-630): after the section's opening line, every
// DataArray until the first line that is not one
u32 read_tags(Reader& r, Mesh& m, u32 dim, char const* section)
{
  std::string line;
  r.seek(section, line);
  u32 n = 0;
  u32 count = m.counts[dim];
  while (r.next_is("<DataArray", line)) {
    ArrayHead h = parse_head(line);
    void* d = r.array(h, count);
    m.add_tag(dim, h.type, h.name.c_str(), h.ncomps, X_NOT, d);
    ++n;
  }
  return n;
}

// read_ents (vtk_io.cpp:662-682)
void read_ents(Reader& r, Mesh& m, u32 ent_dim, u32 nents)
{
  char const* name = ent_dim == m.dim ? "<Cell" : ent_dim == 1 ? "<Edge" : "<Face";
  std::string line;
  r.seek(name, line);
  r.seek("<DataArray", line);
  ArrayHead h = parse_head(line);
  if (h.type != T_U32 || h.name != "connectivity" || h.ncomps != 1)
    io_fail(std::string(name + 1) + " connectivity is not a UInt32 \"connectivity\" array");
  u32 vpe = deg(ent_dim, 0);
  u32* conn = static_cast<u32*>(r.array(h, (u64)nents * vpe));
  // our check, not the reference's: every vertex index names a vertex
  u64 nuses = (u64)nents * vpe;
  if (nuses > 0xffffffffull) {
    dev_free(conn, m.s);
    io_fail(std::string(name + 1) + " connectivity is too long");
  }
  if (nuses && max_u32(conn, (u32)nuses, m.s) >= m.counts[0]) {
    dev_free(conn, m.s);
    io_fail(std::string(name + 1) + " connectivity names a vertex past NumberOfPoints");
  }
  m.set_ents(ent_dim, nents, conn);
}

// mesh_parallel_from_tags (parallel_mesh.cpp:240-262)
void parallel_from_tags(Mesh& m, u32 d)
{
  Tag* g = m.find_tag(d, "global_number");
  if (!g) return;
  if (g->type != T_U64 || g->ncomps != 1) io_fail("global_number is not one UInt64");
  u32 n = m.counts[d];
  u64* gl = dalloc<u64>(n ? n : 1, m.s);
  if (n) CK(cudaMemcpyAsync(gl, g->data, sizeof(u64) * n, cudaMemcpyDeviceToDevice, m.s));
  m.set_globals(d, gl);  // forgets the owners too
  m.remove_tag(d, "global_number");
  char const* names[2] = {"own_rank", "own_id"};
  u32** dst[2] = {&m.own_ranks[d], &m.own_ids[d]};
  for (u32 k = 0; k < 2; ++k) {
    Tag* t = m.find_tag(d, names[k]);
    if (!t) return;
    if (t->type != T_U32 || t->ncomps != 1) io_fail(std::string(names[k]) + " is not one UInt32");
    u32* a = dalloc<u32>(n ? n : 1, m.s);
    if (n) CK(cudaMemcpyAsync(a, t->data, sizeof(u32) * n, cudaMemcpyDeviceToDevice, m.s));
    *dst[k] = a;
    m.remove_tag(d, names[k]);
  }
}

Mesh* read_vtu(char const* path, bool is_parallel)
{
  std::unique_ptr<Mesh> m;
  Reader r(path, nullptr);
  std::string line;
  // read_unstructured_header (vtk_io.cpp:437-452)
  r.seek("<VTKFile", line);
  std::string v;
  bool file_little = host_little_endian();
  if (try_attrib(line, "byte_order", v)) file_little = v == "LittleEndian";
  r.swap = file_little != host_little_endian();
  r.compressed = try_attrib(line, "compressor", v);
  if (try_attrib(line, "header_type", v) && v != "UInt32")
    io_fail("header_type " + v + " is not supported (UInt32 only)");
  // read_piece_header (vtk_io.cpp:468-485)
  r.seek("<Piece", line);
  u32 nverts = (u32)atoi(attrib(line, "NumberOfPoints").c_str());
  u32 nelems = (u32)atoi(attrib(line, "NumberOfCells").c_str());
  u32 nedges = 0, nfaces = 0;
  bool do_edges = try_int_attrib(line, "NumberOfEdges", &nedges);
  bool do_faces = try_int_attrib(line, "NumberOfFaces", &nfaces);
  bool full = try_attrib(line, "Rep", v) && v == "Full";
  if (!nelems) io_fail("the file has no cells");
  // read_dimension (vtk_io.cpp:583-609): the element type of the Cells
  r.seek("<Cells", line);
  for (;;) {
    r.seek("<DataArray", line);
    if (attrib(line, "Name") == "types") break;
  }
  ArrayHead th = parse_head(line);
  if (th.type != T_U8 || th.ncomps != 1) io_fail("cell types are not one UInt8");
  unsigned char* dtypes = static_cast<unsigned char*>(r.array(th, nelems));
  std::vector<unsigned char> types(nelems);
  CK(cudaMemcpyAsync(types.data(), dtypes, nelems, cudaMemcpyDeviceToHost, r.s));
  stream_sync(r.s);
  dev_free(dtypes, r.s);
  u32 dim = 0;
  while (dim < 4 && types[0] != CELL_TYPES[dim]) ++dim;
  if (dim == 4) io_fail("cells are not simplices");
  for (u32 i = 0; i < nelems; ++i)
    if (types[i] != CELL_TYPES[dim]) io_fail("cells of more than one type");
  if (dim == 0) io_fail("a mesh of vertex cells is not supported");
  m.reset(new Mesh(dim, full, is_parallel, nullptr));
  r.s = m->s;
  m->set_ents(0, nverts, nullptr);
  // read_vtk_mesh (vtk_io.cpp:684-703): points, edges, faces, cells
  r.pos = 0;
  if (read_tags(r, *m, 0, "<Points") != 1) io_fail("Points must hold exactly one array");
  if (do_edges) read_ents(r, *m, 1, nedges);
  if (do_faces) read_ents(r, *m, 2, nfaces);
  read_ents(r, *m, dim, nelems);
  // read_vtk_fields (vtk_io.cpp:713-724)
  read_tags(r, *m, 0, "<PointData");
  if (is_parallel) parallel_from_tags(*m, 0);
  if (dim > 1 && m->has_dim(1)) {
    read_tags(r, *m, 1, "<EdgeData");
    if (is_parallel) parallel_from_tags(*m, 1);
  }
  if (dim > 2 && m->has_dim(2)) {
    read_tags(r, *m, 2, "<FaceData");
    if (is_parallel) parallel_from_tags(*m, 2);
  }
  read_tags(r, *m, dim, "<CellData");
  if (is_parallel) parallel_from_tags(*m, dim);
  stream_sync(m->s);
  return m.release();
}

// ---------------------------------------------------------------------------
// writing

struct Writer {
  FILE* f = nullptr;
  cudaStream_t s;
  bool ascii;
  bool compress;
  std::string path;
  // staging: device text and its pinned host copy, grown as needed
  char* dtext = nullptr;
  size_t dcap = 0;
  char* htext = nullptr;
  size_t hcap = 0;
  std::vector<char> iobuf;

  Writer(char const* p, cudaStream_t st, bool asc, bool comp)
      : s(st), ascii(asc), compress(comp), path(p)
  {
    f = fopen(p, "w");
    if (!f) io_fail(std::string("cannot create ") + p + ": " + strerror(errno));
    iobuf.resize(1 << 22);
    setvbuf(f, iobuf.data(), _IOFBF, iobuf.size());
  }
  ~Writer()
  {
    if (f) fclose(f);
    cudaStreamSynchronize(s);
    if (dtext) cudaFreeAsync(dtext, s);
    if (htext) cudaFreeHost(htext);
  }
  void close()
  {
    int bad = ferror(f);
    if (fclose(f) != 0 || bad) {
      f = nullptr;
      io_fail("cannot write " + path);
    }
    f = nullptr;
  }
  void put(char const* str) { fputs(str, f); }

  void* host_staging(size_t n)
  {
    if (n > hcap) {
      if (htext) cudaFreeHost(htext);
      htext = nullptr;
      hcap = 0;
      if (cudaMallocHost(&htext, n) != cudaSuccess) throw Failure(E_NOMEM, "pinned staging");
      hcap = n;
    }
    return htext;
  }

  // write_binary_array (vtk_io.cpp:149-171)
  void binary(u32 nbytes, void const* d)
  {
    if (!compress) {
      std::string head = b64_host(&nbytes, 4);
      fwrite(head.data(), 1, head.size(), f);
      size_t nch = b64_chars(nbytes);
      if (nch) {
        if (nch > dcap) {
          dev_free(dtext, s);
          dtext = dalloc<char>(nch, s);
          dcap = nch;
        }
        CK(launch_kernel(k_b64_encode, dim3(encode_grid(nbytes)), dim3(BLOCK), 0, s, 
            static_cast<unsigned char const*>(d), nbytes, reinterpret_cast<char4*>(dtext)));
        CK_LAUNCH();
        char* h = static_cast<char*>(host_staging(nch));
        CK(cudaMemcpyAsync(h, dtext, nch, cudaMemcpyDeviceToHost, s));
        stream_sync(s);
        fwrite(h, 1, nch, f);
      }
    } else {
      unsigned char* h = static_cast<unsigned char*>(host_staging(nbytes ? nbytes : 1));
      if (nbytes) CK(cudaMemcpyAsync(h, d, nbytes, cudaMemcpyDeviceToHost, s));
      stream_sync(s);
      uLongf csize = compressBound(nbytes);
      std::vector<unsigned char> comp(csize);
      if (::compress(comp.data(), &csize, h, nbytes) != Z_OK) io_fail("zlib compress failed");
      u32 hdr[4] = {1, nbytes, nbytes, (u32)csize};
      std::string head = b64_host(hdr, sizeof(hdr));
      fwrite(head.data(), 1, head.size(), f);
      std::string body = b64_host(comp.data(), csize);
      fwrite(body.data(), 1, body.size(), f);
    }
    fputc('\n', f);
  }

  // write_ascii_array (vtk_io.cpp:220-263)
  void ascii_values(u32 type, u64 nents, u32 ncomps, void const* d)
  {
    size_t nbytes = nents * ncomps * tag_esz(type);
    void* h = host_staging(nbytes ? nbytes : 1);
    if (nbytes) CK(cudaMemcpyAsync(h, d, nbytes, cudaMemcpyDeviceToHost, s));
    stream_sync(s);
    for (u64 i = 0; i < nents; ++i) {
      for (u32 j = 0; j < ncomps; ++j) {
        u64 k = i * ncomps + j;
        switch (type) {
          case T_U8: fprintf(f, " %u", (unsigned)static_cast<unsigned char const*>(h)[k]); break;
          case T_U32: fprintf(f, " %u", static_cast<u32 const*>(h)[k]); break;
          case T_U64: fprintf(f, " %lu", static_cast<u64 const*>(h)[k]); break;
          default: fprintf(f, " %.15e", static_cast<double const*>(h)[k]); break;
        }
      }
      fputc('\n', f);
    }
  }

  // write_array (vtk_io.cpp:319-336)
  void array(u32 type, char const* name, u64 nents, u32 ncomps, void const* d)
  {
    u64 nbytes = nents * ncomps * tag_esz(type);
    if (!ascii && nbytes > 0xffffffffull)
      io_fail(std::string("array ") + name + " exceeds the UInt32 byte count of the format");
    fprintf(f, "<DataArray type=\"%s\" Name=\"%s\" NumberOfComponents=\"%u\" format=\"%s\">\n",
        TYPE_NAMES[type], name, ncomps, ascii ? "ascii" : "binary");
    if (ascii)
      ascii_values(type, nents, ncomps, d);
    else
      binary((u32)nbytes, d);
    fprintf(f, "</DataArray>\n");
  }
};

// the tags a parallel mesh shows while it is written (mesh_parallel_to_tags,
// parallel_mesh.cpp:219-228): its global numbers, and owner ranks / ids
// where they were asked for
struct ParallelTag {
  u32 type;
  char const* name;
  void const* data;
};

std::vector<ParallelTag> parallel_tags(Mesh& m, u32 d)
{
  std::vector<ParallelTag> out;
  if (!m.parallel) return out;
  if (m.has_globals(d)) out.push_back({T_U64, "global_number", m.ask_globals(d)});
  if (m.has_own_ranks(d)) out.push_back({T_U32, "own_rank", m.ask_own_ranks(d)});
  if (m.has_own_ids(d)) out.push_back({T_U32, "own_id", m.ask_own_ids(d)});
  return out;
}

void write_tags(Writer& w, Mesh& m, u32 d, Tag const* except)
{
  u32 n = m.counts[d];
  for (auto const& t : m.tags[d])
    if (&t != except) w.array(t.type, t.name.c_str(), n, t.ncomps, t.data);
  for (auto const& t : parallel_tags(m, d)) w.array(t.type, t.name, n, 1, t.data);
}

void write_connectivity(Writer& w, Mesh& m, u32 d)
{
  u32 const* conn = m.ask_down(d, 0);
  w.array(T_U32, "connectivity", (u64)m.counts[d] * deg(d, 0), 1, conn);
}

// write_vtu_opts (vtk_io.cpp:487-538)
void write_vtu(Mesh& m, char const* path, bool ascii, bool compress)
{
  u32 dim = m.dim;
  Tag* coords = m.find_tag(0, "coordinates");
  if (!coords) throw Failure(E_ARG, "mesh has no coordinates");
  for (u32 d = 1; d <= dim; ++d)
    if (d == dim || m.has_dim(d)) m.ask_down(d, 0);
  bool do_edges = dim > 1 && m.has_dim(1);
  bool do_faces = dim > 2 && m.has_dim(2);
  u32 nelems = m.counts[dim];
  Writer w(path, m.s, ascii, compress);
  w.put("<VTKFile type=\"UnstructuredGrid\"");
  if (!ascii) {
    w.put(host_little_endian() ? " byte_order=\"LittleEndian\"" : " byte_order=\"BigEndian\"");
    w.put(" header_type=\"UInt32\"");
    if (compress) w.put(" compressor=\"vtkZLibDataCompressor\"");
  }
  w.put(">\n<UnstructuredGrid>\n");
  fprintf(w.f, "<Piece NumberOfPoints=\"%u\" NumberOfCells=\"%u\"", m.counts[0], nelems);
  if (do_edges) fprintf(w.f, " NumberOfEdges=\"%u\"", m.counts[1]);
  if (do_faces) fprintf(w.f, " NumberOfFaces=\"%u\"", m.counts[2]);
  fprintf(w.f, " Rep=\"%s\">\n", m.full ? "Full" : "Reduced");
  w.put("<Points>\n");
  w.array(coords->type, coords->name.c_str(), m.counts[0], coords->ncomps, coords->data);
  w.put("</Points>\n");
  if (do_edges) {
    w.put("<Edges>\n");
    write_connectivity(w, m, 1);
    w.put("</Edges>\n");
  }
  if (do_faces) {
    w.put("<Faces>\n");
    write_connectivity(w, m, 2);
    w.put("</Faces>\n");
  }
  w.put("<Cells>\n");
  write_connectivity(w, m, dim);
  {
    u32* offs = dalloc<u32>(nelems ? nelems : 1, m.s);
    unsigned char* types = dalloc<unsigned char>(nelems ? nelems : 1, m.s);
    if (nelems) {
      CK(launch_kernel(k_cell_arrays, dim3(grid_for(nelems)), dim3(BLOCK), 0, m.s, nelems, deg(dim, 0), offs, types,
          CELL_TYPES[dim]));
      CK_LAUNCH();
    }
    try {
      w.array(T_U32, "offsets", nelems, 1, offs);
      w.array(T_U8, "types", nelems, 1, types);
    } catch (...) {
      dev_free(offs, m.s);
      dev_free(types, m.s);
      throw;
    }
    dev_free(offs, m.s);
    dev_free(types, m.s);
  }
  w.put("</Cells>\n<PointData>\n");
  write_tags(w, m, 0, coords);
  w.put("</PointData>\n");
  if (do_edges) {
    w.put("<EdgeData>\n");
    write_tags(w, m, 1, nullptr);
    w.put("</EdgeData>\n");
  }
  if (do_faces) {
    w.put("<FaceData>\n");
    write_tags(w, m, 2, nullptr);
    w.put("</FaceData>\n");
  }
  w.put("<CellData>\n");
  write_tags(w, m, dim, nullptr);
  w.put("</CellData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n");
  w.close();
}

void describe_array(FILE* f, u32 type, char const* name, u32 ncomps)
{
  fprintf(f, "<PDataArray type=\"%s\" Name=\"%s\" NumberOfComponents=\"%u\" format=\"ascii\"/>\n",
      TYPE_NAMES[type], name, ncomps);
}

// write_pvtu (vtk_io.cpp:739-771), one piece
void write_pvtu(Mesh& m, char const* path, std::string const& piece_name)
{
  FILE* f = fopen(path, "w");
  if (!f) io_fail(std::string("cannot create ") + path + ": " + strerror(errno));
  fprintf(f, "<VTKFile type=\"PUnstructuredGrid\">\n");
  fprintf(f, "<PUnstructuredGrid GhostLevel=\"%u\">\n", m.parallel ? m.ghost_layers : 0u);
  Tag* coords = m.find_tag(0, "coordinates");
  fprintf(f, "<PPointData>\n");
  for (auto const& t : m.tags[0])
    if (&t != coords) describe_array(f, t.type, t.name.c_str(), t.ncomps);
  for (auto const& t : parallel_tags(m, 0)) describe_array(f, t.type, t.name, 1);
  fprintf(f, "</PPointData>\n<PCellData>\n");
  for (auto const& t : m.tags[m.dim]) describe_array(f, t.type, t.name.c_str(), t.ncomps);
  for (auto const& t : parallel_tags(m, m.dim)) describe_array(f, t.type, t.name, 1);
  fprintf(f, "</PCellData>\n<PPoints>\n");
  describe_array(f, coords->type, coords->name.c_str(), coords->ncomps);
  fprintf(f, "</PPoints>\n");
  fprintf(f, "<Piece Source=\"%s\"/>\n", piece_name.c_str());
  fprintf(f, "</PUnstructuredGrid>\n</VTKFile>\n");
  int bad = ferror(f);
  if (fclose(f) != 0 || bad) io_fail(std::string("cannot write ") + path);
}

// split_pathname (files.cpp:24-43): the path without its suffix, the suffix
void split_path(char const* path, std::string& prefix, std::string& suffix)
{
  std::string p(path);
  size_t dot = p.rfind('.');
  if (dot == std::string::npos) throw Failure(E_ARG, std::string("no file suffix in ") + path);
  prefix = p.substr(0, dot);
  suffix = p.substr(dot + 1);
}

}  // namespace

// read_mesh_vtk (vtk_io.cpp:787-805) for one rank: "x.vtu" is a serial mesh;
// "x.pvtu" reads its single piece "x.vtu" as a parallel mesh (global
// numbers from the global_number tags) with the GhostLevel of "x.pvtu"
Mesh* read_vtk(char const* path)
{
  if (!path) throw Failure(E_ARG, "null path");
  std::string prefix, suffix;
  split_path(path, prefix, suffix);
  bool is_parallel = suffix == "pvtu";
  std::string piece = prefix + ".vtu";
  Mesh* m = read_vtu(piece.c_str(), is_parallel);
  if (is_parallel) {
    try {
      Reader r(path, m->s);
      std::string line;
      r.seek("<PUnstructuredGrid", line);
      u32 n = 0;
      if (try_int_attrib(line, "GhostLevel", &n)) m->ghost_layers = n;
    } catch (...) {
      delete m;
      throw;
    }
  }
  return m;
}

// write_mesh_vtk_opts (vtk_io.cpp:807-826) for one rank: the piece goes to
// "<prefix>.vtu"; a ".pvtu" path also gets the parallel index file
void write_vtk(Mesh& m, char const* path, bool ascii, bool compress)
{
  if (!path) throw Failure(E_ARG, "null path");
  std::string prefix, suffix;
  split_path(path, prefix, suffix);
  std::string piece = prefix + ".vtu";
  write_vtu(m, piece.c_str(), ascii, compress);
  if (suffix == "pvtu") {
    size_t slash = prefix.rfind('/');
    std::string name = slash == std::string::npos ? prefix : prefix.substr(slash + 1);
    write_pvtu(m, path, name + ".vtu");
  }
}

}  // namespace osh
