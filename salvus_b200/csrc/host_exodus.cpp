// host_exodus.cpp -- Exodus II mesh / model reader without the Exodus or
// NetCDF libraries: a reader of the NetCDF classic container (CDF-1 and the
// 64-bit-offset CDF-2, the formats the Exodus library of the reference's era
// writes by default) and the Exodus II naming conventions on top of it.
//
// What the reference reads (Mesh::read Mesh.cpp:53-86 through
// DMPlexCreateExodusFromFile; ExodusModel::read ExodusModel.cpp:37-81,
// 230-265, 350-379, 524-545):
//   coordinates    coord [num_dim][num_nodes] or coordx / coordy / coordz
//   element blocks connect<b> [num_el_in_blk<b>][num_nod_per_el<b>] (1-based),
//                  attribute elem_type; blocks concatenated in block order
//   elemental vars name_elem_var [num_elem_var][len_name] and
//                  vals_elem_var<v>eb<b> [time_step][num_el_in_blk<b>] (first
//                  time step), per-vertex parameters named NAME_<i>, the
//                  fluid flag named "fluid" (ExodusModel.cpp:422-520)
//   side sets      elem_ss<s>, side_ss<s> (1-based element and side), names
//                  ss_names [num_side_sets][len_name]
// Vertex orders are converted to the library's (PETSc right-hand) orders:
// QUAD4 and TRI3 unchanged, HEX8 bottom face reversed (n0 n3 n2 n1 n4..n7, as
// DMPlexCreateExodus inverts hexahedra), TET4 n0 n2 n1 n3 (positive TetP1
// orientation); parameter NAME_<i> belongs to vertex i of that order, as the
// reference attaches it to the i-th vertex of the DMPlex closure
// (ElementAdapter attachMaterialProperties).
//
// NetCDF-4 files (an HDF5 container) need the HDF5 library, which this build
// does not have; they are rejected with that message.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "internal.h"

struct salvus_exodus {
  // NetCDF classic header
  struct Dim {
    std::string name;
    int64_t len;  // 0: the record dimension
  };
  struct Att {
    std::string name;
    int type;
    int64_t n;
    std::vector<uint8_t> raw;  // big-endian values
  };
  struct Var {
    std::string name;
    std::vector<int64_t> dims;
    std::vector<Att> atts;
    int type;
    int64_t vsize, begin;
    bool record;
  };
  std::string path;
  int version = 0;
  int64_t numrecs = 0, recsize = 0;
  std::vector<Dim> dims;
  std::vector<Att> gatts;
  std::vector<Var> vars;
  // Exodus content
  int shape = -1, dim = 0, nv = 0;
  int64_t n_vertices = 0, n_elements = 0;
  std::vector<double> vertices;     // [n_vertices][dim]
  std::vector<int64_t> cells;       // [n_elements][nv], library vertex order, 0-based
  std::vector<int> order;           // library vertex i = Exodus node order[i]
  std::vector<std::string> var_names;
  std::vector<std::vector<double>> var_vals;  // [n_elem_vars][n_elements]
  std::vector<std::string> ss_names;
  std::vector<std::vector<int64_t>> ss_elem, ss_side;  // 1-based as stored
};

namespace salvus {
namespace {

enum { NC_BYTE = 1, NC_CHAR = 2, NC_SHORT = 3, NC_INT = 4, NC_FLOAT = 5, NC_DOUBLE = 6 };
int type_size(int t) {
  switch (t) {
    case NC_BYTE: case NC_CHAR: return 1;
    case NC_SHORT: return 2;
    case NC_INT: case NC_FLOAT: return 4;
    case NC_DOUBLE: return 8;
  }
  return 0;
}

struct Reader {
  FILE *f = nullptr;
  bool bad = false;
  ~Reader() {
    if (f) std::fclose(f);
  }
  bool read(void *p, size_t n) {
    if (bad || std::fread(p, 1, n, f) != n) bad = true;
    return !bad;
  }
  uint32_t u32() {
    uint8_t b[4] = {0, 0, 0, 0};
    read(b, 4);
    return (uint32_t)b[0] << 24 | (uint32_t)b[1] << 16 | (uint32_t)b[2] << 8 | b[3];
  }
  uint64_t u64() {
    const uint64_t hi = u32();
    return hi << 32 | u32();
  }
  std::string name() {
    const uint32_t n = u32();
    if (bad || n > (1u << 16)) {
      bad = true;
      return {};
    }
    std::string s(n, '\0');
    read(&s[0], n);
    skip_pad(n);
    return s;
  }
  void skip_pad(uint64_t n) {
    const uint64_t pad = (4 - n % 4) % 4;
    uint8_t z[4];
    if (pad) read(z, (size_t)pad);
  }
};

double be_value(const uint8_t *p, int type) {
  switch (type) {
    case NC_BYTE: return (double)(int8_t)p[0];
    case NC_CHAR: return (double)p[0];
    case NC_SHORT: return (double)(int16_t)((uint16_t)p[0] << 8 | p[1]);
    case NC_INT: return (double)(int32_t)((uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]);
    case NC_FLOAT: {
      uint32_t u = (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3];
      float x;
      std::memcpy(&x, &u, 4);
      return (double)x;
    }
    case NC_DOUBLE: {
      uint64_t u = 0;
      for (int k = 0; k < 8; ++k) u = u << 8 | p[k];
      double x;
      std::memcpy(&x, &u, 8);
      return x;
    }
  }
  return 0.0;
}

int parse_atts(Reader &r, std::vector<salvus_exodus::Att> &out) {
  const uint32_t tag = r.u32(), n = r.u32();
  if (tag == 0 && n == 0) return SALVUS_OK;
  if (tag != 0x0C) return fail(SALVUS_E_INVALID, "NetCDF header: attribute list expected");
  for (uint32_t i = 0; i < n && !r.bad; ++i) {
    salvus_exodus::Att a;
    a.name = r.name();
    a.type = (int)r.u32();
    a.n = r.u32();
    const int ts = type_size(a.type);
    if (!ts) return fail(SALVUS_E_INVALID, "NetCDF header: attribute type %d", a.type);
    a.raw.resize((size_t)(a.n * ts));
    if (!a.raw.empty()) r.read(a.raw.data(), a.raw.size());
    r.skip_pad((uint64_t)(a.n * ts));
    out.push_back(std::move(a));
  }
  return r.bad ? fail(SALVUS_E_INVALID, "NetCDF header truncated") : SALVUS_OK;
}

int parse_header(salvus_exodus *x, Reader &r) {
  uint8_t magic[4];
  if (!r.read(magic, 4)) return fail(SALVUS_E_INVALID, "%s: empty file", x->path.c_str());
  if (magic[0] == 0x89 && magic[1] == 'H' && magic[2] == 'D' && magic[3] == 'F')
    return fail(SALVUS_E_UNSUPPORTED,
                "%s is a NetCDF-4 (HDF5) file; this build reads the NetCDF classic formats only "
                "(the HDF5 library is not available)", x->path.c_str());
  if (magic[0] != 'C' || magic[1] != 'D' || magic[2] != 'F' || (magic[3] != 1 && magic[3] != 2))
    return fail(SALVUS_E_INVALID, "%s is not a NetCDF classic (CDF-1 / CDF-2) file",
                x->path.c_str());
  x->version = magic[3];
  x->numrecs = r.u32();
  // dimensions
  uint32_t tag = r.u32(), n = r.u32();
  if (!(tag == 0 && n == 0)) {
    if (tag != 0x0A) return fail(SALVUS_E_INVALID, "NetCDF header: dimension list expected");
    for (uint32_t i = 0; i < n && !r.bad; ++i) {
      salvus_exodus::Dim d;
      d.name = r.name();
      d.len = r.u32();
      x->dims.push_back(d);
    }
  }
  int rc = parse_atts(r, x->gatts);
  if (rc) return rc;
  tag = r.u32();
  n = r.u32();
  if (!(tag == 0 && n == 0)) {
    if (tag != 0x0B) return fail(SALVUS_E_INVALID, "NetCDF header: variable list expected");
    for (uint32_t i = 0; i < n && !r.bad; ++i) {
      salvus_exodus::Var v;
      v.name = r.name();
      const uint32_t nd = r.u32();
      if (nd > 64) return fail(SALVUS_E_INVALID, "NetCDF header: %u dimensions", nd);
      for (uint32_t k = 0; k < nd; ++k) {
        const uint32_t id = r.u32();
        if (id >= x->dims.size()) return fail(SALVUS_E_INVALID, "NetCDF header: dimension id");
        v.dims.push_back(id);
      }
      if ((rc = parse_atts(r, v.atts))) return rc;
      v.type = (int)r.u32();
      if (!type_size(v.type)) return fail(SALVUS_E_INVALID, "NetCDF header: variable type %d", v.type);
      v.vsize = r.u32();
      v.begin = x->version == 1 ? (int64_t)r.u32() : (int64_t)r.u64();
      v.record = !v.dims.empty() && x->dims[(size_t)v.dims[0]].len == 0;
      x->vars.push_back(std::move(v));
    }
  }
  if (r.bad) return fail(SALVUS_E_INVALID, "%s: NetCDF header truncated", x->path.c_str());
  // record size: sum of the record variables' per-record sizes (one record
  // variable of a narrow type is not padded)
  int nrecvars = 0;
  for (auto &v : x->vars) nrecvars += v.record;
  for (auto &v : x->vars)
    if (v.record) {
      int64_t s = type_size(v.type);
      for (size_t k = 1; k < v.dims.size(); ++k) s *= x->dims[(size_t)v.dims[k]].len;
      if (nrecvars > 1) s = (s + 3) / 4 * 4;
      x->recsize += s;
    }
  return SALVUS_OK;
}

const salvus_exodus::Dim *find_dim(const salvus_exodus *x, const std::string &name) {
  for (auto &d : x->dims)
    if (d.name == name) return &d;
  return nullptr;
}
const salvus_exodus::Var *find_var(const salvus_exodus *x, const std::string &name) {
  for (auto &v : x->vars)
    if (v.name == name) return &v;
  return nullptr;
}
int64_t dim_len(const salvus_exodus *x, const std::string &name) {
  const auto *d = find_dim(x, name);
  return d ? d->len : -1;
}

// values of a variable (record variables: the first record), as doubles
int read_var(const salvus_exodus *x, const salvus_exodus::Var &v, std::vector<double> &out) {
  int64_t count = 1;
  for (size_t k = v.record ? 1 : 0; k < v.dims.size(); ++k) count *= x->dims[(size_t)v.dims[k]].len;
  if (v.record && x->numrecs < 1)
    return fail(SALVUS_E_INVALID, "%s: variable %s has no time step", x->path.c_str(), v.name.c_str());
  const int ts = type_size(v.type);
  std::vector<uint8_t> raw((size_t)(count * ts));
  FILE *f = std::fopen(x->path.c_str(), "rb");
  if (!f) return fail(SALVUS_E_INVALID, "cannot reopen %s", x->path.c_str());
  bool ok = std::fseek(f, (long)v.begin, SEEK_SET) == 0 &&
            (raw.empty() || std::fread(raw.data(), 1, raw.size(), f) == raw.size());
  std::fclose(f);
  if (!ok) return fail(SALVUS_E_INVALID, "%s: variable %s lies beyond the end of the file",
                       x->path.c_str(), v.name.c_str());
  out.resize((size_t)count);
  for (int64_t i = 0; i < count; ++i) out[(size_t)i] = be_value(&raw[(size_t)(i * ts)], v.type);
  return SALVUS_OK;
}

int read_named(const salvus_exodus *x, const std::string &name, std::vector<double> &out) {
  const auto *v = find_var(x, name);
  if (!v) return fail(SALVUS_E_NOT_FOUND, "%s: no variable %s", x->path.c_str(), name.c_str());
  return read_var(x, *v, out);
}

// fixed-width character rows of a [n][len] char variable
int read_strings(const salvus_exodus *x, const std::string &name, std::vector<std::string> &out) {
  const auto *v = find_var(x, name);
  out.clear();
  if (!v) return SALVUS_OK;
  if (v->type != NC_CHAR || v->dims.size() != 2)
    return fail(SALVUS_E_INVALID, "%s: %s is not a character table", x->path.c_str(), name.c_str());
  std::vector<double> c;
  int rc = read_var(x, *v, c);
  if (rc) return rc;
  const int64_t rows = x->dims[(size_t)v->dims[0]].len, len = x->dims[(size_t)v->dims[1]].len;
  for (int64_t i = 0; i < rows; ++i) {
    std::string s;
    for (int64_t k = 0; k < len; ++k) {
      const char ch = (char)c[(size_t)(i * len + k)];
      if (ch == '\0') break;
      s.push_back(ch);
    }
    while (!s.empty() && s.back() == ' ') s.pop_back();
    out.push_back(s);
  }
  return SALVUS_OK;
}

std::string att_string(const salvus_exodus::Var &v, const std::string &name) {
  for (auto &a : v.atts)
    if (a.name == name && a.type == NC_CHAR) {
      std::string s(a.raw.begin(), a.raw.end());
      while (!s.empty() && (s.back() == '\0' || s.back() == ' ')) s.pop_back();
      return s;
    }
  return {};
}

int load_exodus(salvus_exodus *x) {
  const int64_t dim = dim_len(x, "num_dim"), nn = dim_len(x, "num_nodes");
  const int64_t ne = dim_len(x, "num_elem"), nb = dim_len(x, "num_el_blk");
  if (dim < 2 || dim > 3 || nn <= 0 || ne <= 0 || nb <= 0)
    return fail(SALVUS_E_INVALID, "%s: not an Exodus II mesh (num_dim / num_nodes / num_elem / "
                "num_el_blk)", x->path.c_str());
  x->dim = (int)dim;
  x->n_vertices = nn;
  x->n_elements = ne;
  // coordinates
  x->vertices.assign((size_t)(nn * dim), 0.0);
  std::vector<double> c;
  int rc;
  if (find_var(x, "coord")) {
    if ((rc = read_named(x, "coord", c))) return rc;
    for (int64_t a = 0; a < dim; ++a)
      for (int64_t i = 0; i < nn; ++i) x->vertices[(size_t)(i * dim + a)] = c[(size_t)(a * nn + i)];
  } else {
    const char *names[3] = {"coordx", "coordy", "coordz"};
    for (int64_t a = 0; a < dim; ++a) {
      if ((rc = read_named(x, names[a], c))) return rc;
      for (int64_t i = 0; i < nn; ++i) x->vertices[(size_t)(i * dim + a)] = c[(size_t)i];
    }
  }
  // element blocks (one element type)
  std::string type;
  for (int64_t b = 1; b <= nb; ++b) {
    const std::string cn = "connect" + std::to_string(b);
    const auto *v = find_var(x, cn);
    if (!v) return fail(SALVUS_E_INVALID, "%s: no %s", x->path.c_str(), cn.c_str());
    std::string t = att_string(*v, "elem_type");
    for (auto &ch : t) ch = (char)std::toupper((unsigned char)ch);
    if (b == 1) type = t;
    else if (t != type)
      return fail(SALVUS_E_UNSUPPORTED, "%s: element blocks of different types (%s, %s)",
                  x->path.c_str(), type.c_str(), t.c_str());
    const int64_t nper = dim_len(x, "num_nod_per_el" + std::to_string(b));
    if (x->shape < 0) {
      if (t.rfind("QUAD", 0) == 0 && nper == 4 && dim == 2) {
        x->shape = SALVUS_QUAD; x->order = {0, 1, 2, 3};
      } else if (t.rfind("HEX", 0) == 0 && nper == 8 && dim == 3) {
        x->shape = SALVUS_HEX; x->order = {0, 3, 2, 1, 4, 5, 6, 7};
      } else if (t.rfind("TRI", 0) == 0 && nper == 3 && dim == 2) {
        x->shape = SALVUS_TRI; x->order = {0, 1, 2};
      } else if (t.rfind("TET", 0) == 0 && nper == 4 && dim == 3) {
        x->shape = SALVUS_TET; x->order = {0, 2, 1, 3};
      } else {
        return fail(SALVUS_E_UNSUPPORTED, "%s: element type %s with %lld nodes in %lld-D",
                    x->path.c_str(), t.c_str(), (long long)nper, (long long)dim);
      }
      x->nv = (int)nper;
    }
    if ((rc = read_var(x, *v, c))) return rc;
    const int64_t nel = (int64_t)c.size() / nper;
    for (int64_t e = 0; e < nel; ++e)
      for (int i = 0; i < x->nv; ++i) {
        const int64_t id = (int64_t)c[(size_t)(e * nper + x->order[(size_t)i])] - 1;
        if (id < 0 || id >= nn)
          return fail(SALVUS_E_INVALID, "%s: node id out of range", x->path.c_str());
        x->cells.push_back(id);
      }
  }
  if ((int64_t)x->cells.size() != ne * x->nv)
    return fail(SALVUS_E_INVALID, "%s: blocks hold %zu nodes, expected %lld", x->path.c_str(),
                x->cells.size(), (long long)(ne * x->nv));
  // elemental variables (first time step), blocks concatenated
  if ((rc = read_strings(x, "name_elem_var", x->var_names))) return rc;
  for (size_t k = 0; k < x->var_names.size(); ++k) {
    std::vector<double> all;
    for (int64_t b = 1; b <= nb; ++b) {
      const std::string vn = "vals_elem_var" + std::to_string(k + 1) + "eb" + std::to_string(b);
      if ((rc = read_named(x, vn, c))) return rc;
      all.insert(all.end(), c.begin(), c.end());
    }
    if ((int64_t)all.size() != ne)
      return fail(SALVUS_E_INVALID, "%s: variable %s has %zu values", x->path.c_str(),
                  x->var_names[k].c_str(), all.size());
    x->var_vals.push_back(std::move(all));
  }
  // side sets
  const int64_t ns = dim_len(x, "num_side_sets");
  if (ns > 0) {
    if ((rc = read_strings(x, "ss_names", x->ss_names))) return rc;
    x->ss_names.resize((size_t)ns);
    for (int64_t s = 1; s <= ns; ++s) {
      std::vector<double> el, sd;
      if ((rc = read_named(x, "elem_ss" + std::to_string(s), el)) ||
          (rc = read_named(x, "side_ss" + std::to_string(s), sd)))
        return rc;
      x->ss_elem.emplace_back(el.begin(), el.end());
      x->ss_side.emplace_back(sd.begin(), sd.end());
    }
  }
  return SALVUS_OK;
}

// Exodus side numbering (local node lists, Exodus node order)
const std::vector<std::vector<int>> &exodus_sides(int shape) {
  static const std::vector<std::vector<int>> quad = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
  static const std::vector<std::vector<int>> tri = {{0, 1}, {1, 2}, {2, 0}};
  static const std::vector<std::vector<int>> hex = {{0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6},
                                                    {0, 4, 7, 3}, {0, 3, 2, 1}, {4, 5, 6, 7}};
  static const std::vector<std::vector<int>> tet = {{0, 1, 3}, {1, 2, 3}, {0, 3, 2}, {0, 2, 1}};
  return shape == SALVUS_QUAD ? quad : shape == SALVUS_TRI ? tri : shape == SALVUS_HEX ? hex : tet;
}

int find_name(const std::vector<std::string> &names, const std::string &n) {
  for (size_t i = 0; i < names.size(); ++i)
    if (names[i] == n) return (int)i;
  return -1;
}

}  // namespace
}  // namespace salvus

using namespace salvus;

int salvus_exodus_open(const char *path, salvus_exodus **out) {
  if (!path || !out) return fail(SALVUS_E_INVALID, "null argument");
  *out = nullptr;
  std::unique_ptr<salvus_exodus> x(new salvus_exodus());
  x->path = path;
  Reader r;
  r.f = std::fopen(path, "rb");
  if (!r.f) return fail(SALVUS_E_NOT_FOUND, "cannot open %s", path);
  int rc = parse_header(x.get(), r);
  if (rc) return rc;
  if ((rc = load_exodus(x.get()))) return rc;
  *out = x.release();
  return SALVUS_OK;
}

int salvus_exodus_close(salvus_exodus *x) {
  delete x;
  return SALVUS_OK;
}

int salvus_exodus_info(const salvus_exodus *x, int32_t *shape, int32_t *dim, int64_t *n_vertices,
                       int64_t *n_elements, int32_t *n_elem_vars, int32_t *n_side_sets) {
  if (!x) return fail(SALVUS_E_INVALID, "null file");
  if (shape) *shape = x->shape;
  if (dim) *dim = x->dim;
  if (n_vertices) *n_vertices = x->n_vertices;
  if (n_elements) *n_elements = x->n_elements;
  if (n_elem_vars) *n_elem_vars = (int32_t)x->var_names.size();
  if (n_side_sets) *n_side_sets = (int32_t)x->ss_names.size();
  return SALVUS_OK;
}

int salvus_exodus_mesh(const salvus_exodus *x, double *vertices, int64_t *cells) {
  if (!x) return fail(SALVUS_E_INVALID, "null file");
  if (vertices) std::memcpy(vertices, x->vertices.data(), sizeof(double) * x->vertices.size());
  if (cells) std::memcpy(cells, x->cells.data(), sizeof(int64_t) * x->cells.size());
  return SALVUS_OK;
}

static int copy_name(const std::string &s, char *buf, int32_t len) {
  if (!buf || len <= 0) return fail(SALVUS_E_INVALID, "null buffer");
  std::snprintf(buf, (size_t)len, "%s", s.c_str());
  return (int32_t)s.size() >= len ? fail(SALVUS_E_INVALID, "name longer than the buffer") : SALVUS_OK;
}

int salvus_exodus_variable_name(const salvus_exodus *x, int32_t i, char *buf, int32_t len) {
  if (!x || i < 0 || i >= (int32_t)x->var_names.size()) return fail(SALVUS_E_INVALID, "bad variable index");
  return copy_name(x->var_names[(size_t)i], buf, len);
}

int salvus_exodus_side_set_name(const salvus_exodus *x, int32_t i, char *buf, int32_t len) {
  if (!x || i < 0 || i >= (int32_t)x->ss_names.size()) return fail(SALVUS_E_INVALID, "bad side set index");
  return copy_name(x->ss_names[(size_t)i], buf, len);
}

int salvus_exodus_variable(const salvus_exodus *x, const char *name, double *vals) {
  if (!x || !name || !vals) return fail(SALVUS_E_INVALID, "null argument");
  const int k = find_name(x->var_names, name);
  if (k < 0) return fail(SALVUS_E_NOT_FOUND, "%s: no elemental variable %s", x->path.c_str(), name);
  std::memcpy(vals, x->var_vals[(size_t)k].data(), sizeof(double) * (size_t)x->n_elements);
  return SALVUS_OK;
}

int salvus_exodus_params(const salvus_exodus *x, int32_t physics, double *params) {
  if (!x || !params) return fail(SALVUS_E_INVALID, "null argument");
  const int64_t E = x->n_elements;
  const int nv = x->nv;
  // per-vertex parameter NAME_<i> (ExodusModel.cpp:439-470: VP falls back to
  // VPV and VPV to VP)
  auto vertex_param = [&](const std::string &nm, double *out, const char *need) -> int {
    std::string n = nm;
    if (find_name(x->var_names, n + "_0") < 0) {
      if (n == "VP" && find_name(x->var_names, "VPV_0") >= 0) n = "VPV";
      else if (n == "VS" && find_name(x->var_names, "VSV_0") >= 0) n = "VSV";
      else if (!need) {
        for (int64_t i = 0; i < E * nv; ++i) out[i] = 0.0;
        return SALVUS_OK;
      } else {
        return fail(SALVUS_E_NOT_FOUND, "%s: %s needs elemental variables %s_0..%s_%d",
                    x->path.c_str(), need, nm.c_str(), nm.c_str(), nv - 1);
      }
    }
    for (int i = 0; i < nv; ++i) {
      const int k = find_name(x->var_names, n + "_" + std::to_string(i));
      if (k < 0) return fail(SALVUS_E_NOT_FOUND, "%s: no elemental variable %s_%d", x->path.c_str(), n.c_str(), i);
      for (int64_t e = 0; e < E; ++e) out[e * nv + i] = x->var_vals[(size_t)k][(size_t)e];
    }
    return SALVUS_OK;
  };
  int rc;
  const size_t blk = (size_t)(E * nv);
  switch (physics) {
    case SALVUS_ACOUSTIC:
      return vertex_param("VP", params, "acoustic physics");
    case SALVUS_ELASTIC3D: {
      if ((rc = vertex_param("RHO", params, "elastic physics")) ||
          (rc = vertex_param("VP", params + blk, "elastic physics")) ||
          (rc = vertex_param("VS", params + 2 * blk, "elastic physics")))
        return rc;
      // the library's 3-D elastic physics is isotropic: VPH, VSH, ETA (if
      // present) must agree with VPV, VSV, 1 (Elastic3D.cpp:33-54)
      std::vector<double> t(blk);
      const char *pairs[3][2] = {{"VPH", "VP"}, {"VSH", "VS"}, {"ETA", nullptr}};
      for (int k = 0; k < 3; ++k) {
        if (find_name(x->var_names, std::string(pairs[k][0]) + "_0") < 0) continue;
        if ((rc = vertex_param(pairs[k][0], t.data(), "elastic physics"))) return rc;
        const double *ref = k == 0 ? params + blk : k == 1 ? params + 2 * blk : nullptr;
        for (size_t i = 0; i < blk; ++i)
          if (t[i] != (ref ? ref[i] : 1.0))
            return fail(SALVUS_E_UNSUPPORTED, "%s: anisotropic elastic model (%s differs); read "
                        "it with salvus_exodus_elastic3d_params for a SALVUS_MESH_ELASTIC_TI mesh",
                        x->path.c_str(), pairs[k][0]);
      }
      return SALVUS_OK;
    }
    case SALVUS_ELASTIC2D: {
      const char *names[5] = {"RHO", "C11", "C13", "C33", "C55"};
      for (int k = 0; k < 5; ++k)
        if ((rc = vertex_param(names[k], params + k * blk, "elastic 2-D physics"))) return rc;
      return SALVUS_OK;
    }
    case SALVUS_COUPLED2D: {
      const int kf = find_name(x->var_names, "fluid");
      if (kf < 0)
        return fail(SALVUS_E_NOT_FOUND, "%s: fluid flag not found (ExodusModel.cpp:482-489)",
                    x->path.c_str());
      for (int64_t e = 0; e < E; ++e)
        for (int i = 0; i < nv; ++i) params[e * nv + i] = x->var_vals[(size_t)kf][(size_t)e];
      const char *names[6] = {"VP", "RHO", "C11", "C13", "C33", "C55"};
      for (int k = 0; k < 6; ++k)
        if ((rc = vertex_param(names[k], params + (k + 1) * blk, nullptr))) return rc;
      return SALVUS_OK;
    }
  }
  return fail(SALVUS_E_INVALID, "unknown physics %d", physics);
}

int salvus_exodus_elastic3d_params(const salvus_exodus *x, double *params) {
  if (!x || !params) return fail(SALVUS_E_INVALID, "null argument");
  const size_t blk = (size_t)(x->n_elements * x->nv);
  // per-vertex NAME_<i> (ExodusModel.cpp:439-470), VPV <-> VP and VSV <-> VS
  // fallbacks as in the reference
  auto read = [&](const char *name, const char *alt, double *out, double dflt, bool need) -> int {
    std::string n = name;
    if (find_name(x->var_names, n + "_0") < 0) {
      if (alt && find_name(x->var_names, std::string(alt) + "_0") >= 0) {
        n = alt;
      } else if (!need) {
        for (size_t i = 0; i < blk; ++i) out[i] = dflt;
        return SALVUS_OK;
      } else {
        return fail(SALVUS_E_NOT_FOUND, "%s: elastic physics needs elemental variables %s_0..%s_%d",
                    x->path.c_str(), name, name, x->nv - 1);
      }
    }
    for (int i = 0; i < x->nv; ++i) {
      const int k = find_name(x->var_names, n + "_" + std::to_string(i));
      if (k < 0)
        return fail(SALVUS_E_NOT_FOUND, "%s: no elemental variable %s_%d", x->path.c_str(), n.c_str(), i);
      for (int64_t e = 0; e < x->n_elements; ++e)
        out[e * x->nv + i] = x->var_vals[(size_t)k][(size_t)e];
    }
    return SALVUS_OK;
  };
  int rc;
  if ((rc = read("RHO", nullptr, params, 0.0, true)) ||
      (rc = read("VPV", "VP", params + blk, 0.0, true)) ||
      (rc = read("VSV", "VS", params + 3 * blk, 0.0, true)))
    return rc;
  // horizontal velocities default to the vertical ones, ETA to 1 (isotropic)
  if (find_name(x->var_names, "VPH_0") >= 0) {
    if ((rc = read("VPH", nullptr, params + 2 * blk, 0.0, true))) return rc;
  } else {
    std::copy(params + blk, params + 2 * blk, params + 2 * blk);
  }
  if (find_name(x->var_names, "VSH_0") >= 0) {
    if ((rc = read("VSH", nullptr, params + 4 * blk, 0.0, true))) return rc;
  } else {
    std::copy(params + 3 * blk, params + 4 * blk, params + 4 * blk);
  }
  return read("ETA", nullptr, params + 5 * blk, 1.0, false);
}

int salvus_exodus_side_set_nodes(const salvus_exodus *x, const salvus_mesh *m, const char *name,
                                 int64_t *count, int64_t *nodes) {
  if (!x || !m || !name || !count) return fail(SALVUS_E_INVALID, "null argument");
  const int s = find_name(x->ss_names, name);
  if (s < 0) return fail(SALVUS_E_NOT_FOUND, "%s: no side set %s", x->path.c_str(), name);
  if (m->E != x->n_elements || m->shape != x->shape)
    return fail(SALVUS_E_INVALID, "mesh was not built from this file");
  const int nv = m->nv, P = m->P;
  // Exodus node -> library vertex index
  std::vector<int> lib_of(nv);
  for (int i = 0; i < nv; ++i) lib_of[(size_t)x->order[(size_t)i]] = i;
  const auto &sides = exodus_sides(x->shape);
  // element points of each side: P1 weights vanish on every vertex off the side
  std::vector<std::vector<int>> side_pts(sides.size());
  for (size_t f = 0; f < sides.size(); ++f) {
    std::vector<char> on(nv, 0);
    for (int node : sides[f]) on[(size_t)lib_of[(size_t)node]] = 1;
    for (int q = 0; q < P; ++q) {
      double ref[3], w[8];
      point_ref(m->basis, q, ref);
      p1_weights(m->shape, ref, w);
      bool ok = true;
      for (int v = 0; v < nv && ok; ++v)
        if (!on[(size_t)v] && std::fabs(w[v]) > 1e-12) ok = false;
      if (ok) side_pts[f].push_back(q);
    }
  }
  std::vector<char> flag((size_t)m->G, 0);
  const auto &el = x->ss_elem[(size_t)s], &sd = x->ss_side[(size_t)s];
  for (size_t k = 0; k < el.size(); ++k) {
    const int64_t e = el[k] - 1, side = sd[k] - 1;
    if (e < 0 || e >= m->E || side < 0 || side >= (int64_t)sides.size())
      return fail(SALVUS_E_INVALID, "%s: side set %s entry %zu out of range", x->path.c_str(), name, k);
    for (int q : side_pts[(size_t)side]) flag[(size_t)m->conn[(size_t)(e * P + q)]] = 1;
  }
  int64_t n = 0;
  for (int64_t g = 0; g < m->G; ++g)
    if (flag[(size_t)g]) {
      if (nodes) nodes[n] = g;
      ++n;
    }
  *count = n;
  return SALVUS_OK;
}
