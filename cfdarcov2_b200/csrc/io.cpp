// Output files of the reference's IO layer (include/io_operators_tmpl.hpp)
// written without VTK or nlohmann::json: the .vti image of a field
// (store_history) and mesh.json (store_mesh).  Host only; the caller brings
// the field to host memory (the facade's Variable::host()).
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "cfdb_internal.hpp"

namespace {

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

int open_out(File& file, const char* path, const char* fn) {
  if (!path || !*path) return cfdb_fail(nullptr, CFDB_EINVAL, "%s: empty path", fn);
  file.f = fopen(path, "wb");
  if (!file.f) return cfdb_fail(nullptr, CFDB_EIO, "%s: cannot open %s: %s", fn, path, strerror(errno));
  setvbuf(file.f, nullptr, _IOFBF, 1 << 20);
  return CFDB_OK;
}

int close_out(File& file, const char* path, const char* fn) {
  const bool bad = ferror(file.f) != 0;
  const int rc = fclose(file.f);
  file.f = nullptr;
  if (bad || rc != 0) return cfdb_fail(nullptr, CFDB_EIO, "%s: writing %s failed", fn, path);
  return CFDB_OK;
}

bool dims_ok(int64_t nx, int64_t ny, int64_t nz) {
  return nx >= 1 && ny >= 1 && nz >= 1 && nx <= (1 << 20) && ny <= (1 << 20) && nz <= (1 << 20) &&
         nx * ny * nz <= (int64_t(1) << 33);
}

// JSON-safe array name: letters, digits, '_', '-', '.' kept, anything else '_'
std::string clean_name(const char* name) {
  std::string s = (name && *name) ? name : "field";
  for (char& c : s)
    if (!(isalnum(static_cast<unsigned char>(c)) || c == '_' || c == '-' || c == '.')) c = '_';
  return s;
}

}  // namespace

extern "C" int cfdb_write_vti(const char* path, const char* name, int64_t nx, int64_t ny, int64_t nz,
                              const float* values) {
  const char* fn = "cfdb_write_vti";
  if (!values || !dims_ok(nx, ny, nz)) return cfdb_fail(nullptr, CFDB_EINVAL, "%s: bad dimensions or NULL values", fn);
  const int64_t n = nx * ny * nz;
  // reference cell order (z fastest) -> VTK image point order (x fastest)
  std::vector<float> img;
  try {
    img.resize(size_t(n));
  } catch (const std::bad_alloc&) {
    return cfdb_fail(nullptr, CFDB_ENOMEM, "%s: host allocation failed", fn);
  }
  float lo = values[0], hi = values[0];
  for (int64_t x = 0; x < nx; ++x)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t z = 0; z < nz; ++z) {
        const float v = values[nz * ny * x + nz * y + z];
        img[size_t(x + nx * (y + ny * z))] = v;
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
      }
  const std::string nm = clean_name(name);
  File file;
  if (int rc = open_out(file, path, fn)) return rc;
  FILE* f = file.f;
  const long long X = nx - 1, Y = ny - 1, Z = nz - 1;
  fprintf(f, "<?xml version=\"1.0\"?>\n");
  fprintf(f, "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n");
  fprintf(f, "  <ImageData WholeExtent=\"0 %lld 0 %lld 0 %lld\" Origin=\"0 0 0\" Spacing=\"1 1 1\" "
             "Direction=\"1 0 0 0 1 0 0 0 1\">\n", X, Y, Z);
  fprintf(f, "    <Piece Extent=\"0 %lld 0 %lld 0 %lld\">\n", X, Y, Z);
  fprintf(f, "      <PointData Scalars=\"%s\">\n", nm.c_str());
  fprintf(f, "        <DataArray type=\"Float32\" Name=\"%s\" format=\"appended\" RangeMin=\"%.9g\" "
             "RangeMax=\"%.9g\" offset=\"0\"/>\n", nm.c_str(), double(lo), double(hi));
  fprintf(f, "      </PointData>\n      <CellData>\n      </CellData>\n    </Piece>\n  </ImageData>\n");
  fprintf(f, "  <AppendedData encoding=\"raw\">\n   _");
  const uint64_t bytes = uint64_t(n) * sizeof(float);
  fwrite(&bytes, sizeof(bytes), 1, f);  // little-endian host (x86-64, aarch64)
  fwrite(img.data(), sizeof(float), size_t(n), f);
  fprintf(f, "\n  </AppendedData>\n</VTKFile>\n");
  return close_out(file, path, fn);
}

extern "C" int cfdb_write_mesh_json(const char* path, int64_t nx, int64_t ny, int64_t nz, double dx, double dy,
                                    double dz, const double* vertices) {
  const char* fn = "cfdb_write_mesh_json";
  if (!dims_ok(nx, ny, nz) || !(dx > 0) || !(dy > 0) || !(dz > 0))
    return cfdb_fail(nullptr, CFDB_EINVAL, "%s: bad dimensions or spacings", fn);
  const int64_t X = nx, Y = ny, Z = nz;
  // numbering of Mesh3D::init_basic_internals / square_node_coord_to_* (src/mesh3d.cpp:323-416)
  auto vid = [&](int64_t x, int64_t y, int64_t z) { return x * (Z + 1) * (Y + 1) + y * (Z + 1) + z; };
  auto cid = [&](int64_t x, int64_t y, int64_t z) { return Z * Y * x + Z * y + z; };
  const int64_t zf0 = 0, yf0 = X * Y * (Z + 1), xf0 = yf0 + X * (Y + 1) * Z;
  auto fz = [&](int64_t x, int64_t y, int64_t z) { return zf0 + (Z + 1) * Y * x + (Z + 1) * y + z; };
  auto fy = [&](int64_t x, int64_t y, int64_t z) { return yf0 + X * (Y + 1) * z + (Y + 1) * x + y; };
  auto fx = [&](int64_t x, int64_t y, int64_t z) { return xf0 + (X + 1) * Z * y + (X + 1) * z + x; };

  File file;
  if (int rc = open_out(file, path, fn)) return rc;
  FILE* f = file.f;
  // vertexes (Vertex3D holds float coordinates)
  fprintf(f, "{\n    \"vertexes\": [\n");
  for (int64_t x = 0; x <= X; ++x)
    for (int64_t y = 0; y <= Y; ++y)
      for (int64_t z = 0; z <= Z; ++z) {
        const int64_t v = vid(x, y, z);
        // the reference computes x_ * _dx in float (src/mesh3d.cpp:328)
        float c[3] = {float(x) * float(dx), float(y) * float(dy), float(z) * float(dz)};
        if (vertices)
          for (int d = 0; d < 3; ++d) c[d] = float(vertices[3 * v + d]);
        fprintf(f, "        [%.9g, %.9g, %.9g]%s\n", double(c[0]), double(c[1]), double(c[2]),
                (x == X && y == Y && z == Z) ? "" : ",");
      }
  // faces in index order: z faces (x, y, z'), then y faces (z, x, y'), then x faces (y, z, x');
  // each face's corners as its lower cell sets them, cells listed in the cells' loop order
  fprintf(f, "    ],\n    \"face\": [\n");
  const int64_t nfaces = xf0 + (X + 1) * Y * Z;
  int64_t written = 0;
  auto face = [&](int64_t a, int64_t b, int64_t c, int64_t d, int64_t n0, int64_t n1) {
    ++written;
    if (n1 >= 0)
      fprintf(f, "        {\"vertexes_id\": [%lld, %lld, %lld, %lld], \"nodes_id\": [%lld, %lld]}%s\n", (long long)a,
              (long long)b, (long long)c, (long long)d, (long long)n0, (long long)n1, written == nfaces ? "" : ",");
    else
      fprintf(f, "        {\"vertexes_id\": [%lld, %lld, %lld, %lld], \"nodes_id\": [%lld]}%s\n", (long long)a,
              (long long)b, (long long)c, (long long)d, (long long)n0, written == nfaces ? "" : ",");
  };
  for (int64_t x = 0; x < X; ++x)
    for (int64_t y = 0; y < Y; ++y)
      for (int64_t z = 0; z <= Z; ++z)  // plane z: corners (x..x+1, y..y+1, z)
        face(vid(x, y, z), vid(x, y + 1, z), vid(x + 1, y + 1, z), vid(x + 1, y, z), z > 0 ? cid(x, y, z - 1) : cid(x, y, z),
             (z > 0 && z < Z) ? cid(x, y, z) : -1);
  for (int64_t z = 0; z < Z; ++z)
    for (int64_t x = 0; x < X; ++x)
      for (int64_t y = 0; y <= Y; ++y)  // plane y: corners (x..x+1, y, z..z+1)
        face(vid(x, y, z), vid(x, y, z + 1), vid(x + 1, y, z + 1), vid(x + 1, y, z), y > 0 ? cid(x, y - 1, z) : cid(x, y, z),
             (y > 0 && y < Y) ? cid(x, y, z) : -1);
  for (int64_t y = 0; y < Y; ++y)
    for (int64_t z = 0; z < Z; ++z)
      for (int64_t x = 0; x <= X; ++x)  // plane x: corners (x, y..y+1, z..z+1)
        face(vid(x, y, z + 1), vid(x, y + 1, z + 1), vid(x, y + 1, z), vid(x, y, z), x > 0 ? cid(x - 1, y, z) : cid(x, y, z),
             (x > 0 && x < X) ? cid(x, y, z) : -1);
  // nodes: the eight corners and the six faces (z-, z+, y-, y+, x-, x+)
  fprintf(f, "    ],\n    \"nodes\": [\n");
  for (int64_t x = 0; x < X; ++x)
    for (int64_t y = 0; y < Y; ++y)
      for (int64_t z = 0; z < Z; ++z) {
        const long long v[8] = {vid(x, y, z),         vid(x, y, z + 1),         vid(x, y + 1, z),
                                vid(x, y + 1, z + 1), vid(x + 1, y, z),         vid(x + 1, y, z + 1),
                                vid(x + 1, y + 1, z), vid(x + 1, y + 1, z + 1)};
        const long long fc[6] = {fz(x, y, z), fz(x, y, z + 1), fy(x, y, z), fy(x, y + 1, z), fx(x, y, z), fx(x + 1, y, z)};
        fprintf(f, "        {\"vertexes\": [%lld, %lld, %lld, %lld, %lld, %lld, %lld, %lld], "
                   "\"face\": [%lld, %lld, %lld, %lld, %lld, %lld]}%s\n",
                v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], fc[0], fc[1], fc[2], fc[3], fc[4], fc[5],
                (x == X - 1 && y == Y - 1 && z == Z - 1) ? "" : ",");
      }
  fprintf(f, "    ],\n");
  fprintf(f, "    \"x\": %lld,\n    \"y\": %lld,\n    \"z\": %lld,\n", (long long)X, (long long)Y, (long long)Z);
  fprintf(f, "    \"lx\": %.9g,\n    \"ly\": %.9g,\n    \"lz\": %.9g\n}\n", double(float(dx) * float(X)),
          double(float(dy) * float(Y)), double(float(dz) * float(Z)));
  return close_out(file, path, fn);
}

// ---- checkpoints -------------------------------------------------------------
// Header (little-endian, 64 bytes): magic "CFDBCKPT", u32 version, i32 dtype,
// i64 nx, ny, nz, i32 fields, i32 reserved, i64 step, f64 t; then fields x n
// values of the dtype in field order and reference cell order.
namespace {
constexpr char kCkptMagic[8] = {'C', 'F', 'D', 'B', 'C', 'K', 'P', 'T'};
constexpr uint32_t kCkptVersion = 1;

struct CkptHeader {
  char magic[8];
  uint32_t version;
  int32_t dtype;
  int64_t nx, ny, nz;
  int32_t fields, reserved;
  int64_t step;
  double t;
};
static_assert(sizeof(CkptHeader) == 64, "checkpoint header is 64 bytes");

int ckpt_args(const char* fn, int dtype, int64_t nx, int64_t ny, int64_t nz, int32_t fields, const void* data) {
  if (!data || !dims_ok(nx, ny, nz) || fields < 1 || fields > 64 || (dtype != CFDB_F32 && dtype != CFDB_F64))
    return cfdb_fail(nullptr, CFDB_EINVAL, "%s: bad dtype, dimensions, field count or NULL data", fn);
  return CFDB_OK;
}
}  // namespace

extern "C" int cfdb_state_save(const char* path, int dtype, int64_t nx, int64_t ny, int64_t nz, int32_t fields,
                               int64_t step, double t, const void* host_data) {
  const char* fn = "cfdb_state_save";
  if (int rc = ckpt_args(fn, dtype, nx, ny, nz, fields, host_data)) return rc;
  CkptHeader h{};
  std::memcpy(h.magic, kCkptMagic, 8);
  h.version = kCkptVersion;
  h.dtype = dtype;
  h.nx = nx; h.ny = ny; h.nz = nz;
  h.fields = fields;
  h.step = step;
  h.t = t;
  const size_t bytes = size_t(fields) * size_t(nx * ny * nz) * (dtype == CFDB_F64 ? 8 : 4);
  // written to a temporary name and renamed, so an interrupted save never
  // leaves a truncated checkpoint under the final name
  const std::string tmp = std::string(path ? path : "") + ".tmp";
  File file;
  if (int rc = open_out(file, path ? tmp.c_str() : nullptr, fn)) return rc;
  fwrite(&h, sizeof(h), 1, file.f);
  fwrite(host_data, 1, bytes, file.f);
  if (int rc = close_out(file, tmp.c_str(), fn)) {
    std::remove(tmp.c_str());
    return rc;
  }
  if (std::rename(tmp.c_str(), path) != 0) {
    std::remove(tmp.c_str());
    return cfdb_fail(nullptr, CFDB_EIO, "%s: cannot rename %s to %s: %s", fn, tmp.c_str(), path, strerror(errno));
  }
  return CFDB_OK;
}

extern "C" int cfdb_state_load(const char* path, int dtype, int64_t nx, int64_t ny, int64_t nz, int32_t fields,
                               int64_t* step, double* t, void* host_data) {
  const char* fn = "cfdb_state_load";
  if (int rc = ckpt_args(fn, dtype, nx, ny, nz, fields, host_data)) return rc;
  if (!path || !*path) return cfdb_fail(nullptr, CFDB_EINVAL, "%s: empty path", fn);
  File file;
  file.f = fopen(path, "rb");
  if (!file.f) return cfdb_fail(nullptr, CFDB_EIO, "%s: cannot open %s: %s", fn, path, strerror(errno));
  CkptHeader h{};
  if (fread(&h, sizeof(h), 1, file.f) != 1 || std::memcmp(h.magic, kCkptMagic, 8) != 0 || h.version != kCkptVersion)
    return cfdb_fail(nullptr, CFDB_EIO, "%s: %s is not a version-%u checkpoint", fn, path, kCkptVersion);
  if (h.dtype != dtype || h.nx != nx || h.ny != ny || h.nz != nz || h.fields != fields)
    return cfdb_fail(nullptr, CFDB_EINVAL,
                     "%s: %s holds dtype %d, %lld x %lld x %lld cells, %d fields; asked for dtype %d, "
                     "%lld x %lld x %lld, %d fields",
                     fn, path, h.dtype, (long long)h.nx, (long long)h.ny, (long long)h.nz, h.fields, dtype,
                     (long long)nx, (long long)ny, (long long)nz, fields);
  const size_t bytes = size_t(fields) * size_t(nx * ny * nz) * (dtype == CFDB_F64 ? 8 : 4);
  if (fread(host_data, 1, bytes, file.f) != bytes)
    return cfdb_fail(nullptr, CFDB_EIO, "%s: %s is truncated", fn, path);
  if (step) *step = h.step;
  if (t) *t = h.t;
  return CFDB_OK;
}
