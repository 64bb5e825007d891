// cas_reader.cpp -- Fluent ASCII .cas mesh reader: the face-list mesh the
// C-ABI takes (MgpuMesh), read in the library so that a caller without a
// Fortran front end (a server, a test, a Python host) loads a case file
// directly. Host code only.
//
// Follows the record handling of read_cas (mod_uns_cas_reader.f90:44-523):
//   * tokens are "(", ")", quoted strings and whitespace-separated words;
//     a section starts with "(" and its number; unknown sections are skipped
//     to their matching ")";
//   * integers are hexadecimal (decimal when a token is not valid hex);
//   * (10 (zone first last type [dim]) (coords)): zone 0 or type 0 declares
//     the node count only; dim defaults to 2, a 2-D node has z = 0;
//   * (12 (zone first last type [elem]) ...): a data record (zone != 0)
//     raises the cell count to last;
//   * (13 (zone first last bc ftype) (faces)): zone 0 or bc 0 is a
//     declaration, a record without an integer face type a definition; face
//     type 2, 3, 4 is the node count, 5 is followed by the count, 0 means
//     each face leads with its own type; a face lists its nodes, then c0 c1;
//     faces are stored at their own indices first..last;
//   * (45 (zone type name) ()): the zone's type word is kept as its name;
//   * the mesh is rejected when a section is missing or a face refers to a
//     node or cell out of range.

#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/mixgpu.h"

struct MgpuCasMesh {
  std::vector<double> x;  // 3 per node
  std::vector<int32_t> fnode_ptr, fnodes, c0, c1, zone;
  int32_t nnodes = 0, nfaces = 0, ncells = 0;
  std::map<int, std::string> zone_names;
  std::string names_text;  // "id name\n" lines, for mgpu_cas_zone_names
};

namespace {

struct Tokens {
  std::vector<std::string> t;
  size_t p = 0;
  bool end() const { return p >= t.size(); }
};

void tokenize(const std::string& s, std::vector<std::string>& out) {
  size_t i = 0, n = s.size();
  while (i < n) {
    const char ch = s[i];
    if (std::isspace((unsigned char)ch)) {
      ++i;
    } else if (ch == '(' || ch == ')') {
      out.emplace_back(1, ch);
      ++i;
    } else if (ch == '"') {
      size_t j = s.find('"', i + 1);
      if (j == std::string::npos) j = n - 1;
      out.push_back(s.substr(i, j - i + 1));
      i = j + 1;
    } else {
      size_t j = i;
      while (j < n && !std::isspace((unsigned char)s[j]) && s[j] != '(' && s[j] != ')' && s[j] != '"') ++j;
      out.push_back(s.substr(i, j - i));
      i = j;
    }
  }
}

// hexadecimal integer, else decimal; false if neither
bool to_int(const std::string& w, long& v) {
  if (w.empty()) return false;
  char* e = nullptr;
  v = std::strtol(w.c_str(), &e, 16);
  if (e && *e == '\0') return true;
  v = std::strtol(w.c_str(), &e, 10);
  return e && *e == '\0';
}

bool to_real(const std::string& w, double& v) {
  std::string s = w;
  for (auto& ch : s)
    if (ch == 'd' || ch == 'D') ch = 'e';  // Fortran exponent letter
  char* e = nullptr;
  v = std::strtod(s.c_str(), &e);
  return !s.empty() && e && *e == '\0';
}

// From just after a section's "(" + number: skip to the matching ")".
void skip_record(Tokens& T) {
  int depth = 1;
  while (!T.end() && depth > 0) {
    const std::string& w = T.t[T.p++];
    if (w == "(") ++depth;
    else if (w == ")") --depth;
  }
}

// "(" word* ")" at the cursor: the words; false if the cursor is not at "(".
bool read_group(Tokens& T, std::vector<std::string>& g) {
  g.clear();
  if (T.end() || T.t[T.p] != "(") return false;
  ++T.p;
  while (!T.end() && T.t[T.p] != ")") {
    if (T.t[T.p] == "(") return false;  // nested group: not a flat record
    g.push_back(T.t[T.p++]);
  }
  if (T.end()) return false;
  ++T.p;
  return true;
}

struct FaceRec {
  std::vector<int32_t> nodes;
  int32_t c0 = 0, c1 = 0, zone = 0;
  bool set = false;
};

int sec_nodes(Tokens& T, MgpuCasMesh& m) {
  std::vector<std::string> h, c;
  if (!read_group(T, h) || h.size() < 4) return 6;
  long v[5] = {0, 0, 0, 0, 2};
  for (size_t k = 0; k < h.size() && k < 5; ++k)
    if (!to_int(h[k], v[k])) return 6;
  const long zid = v[0], first = v[1], last = v[2], act = v[3], nd = h.size() >= 5 ? v[4] : 2;
  if (last > m.nnodes) {
    m.nnodes = (int32_t)last;
    m.x.resize(3 * (size_t)m.nnodes, 0.0);
  }
  if (zid == 0 || act == 0) {  // declaration
    skip_record(T);
    return 0;
  }
  if (nd < 1 || nd > 3 || first < 1 || last < first) return 7;
  if (!read_group(T, c) || c.size() < (size_t)((last - first + 1) * nd)) return 7;
  for (long i = 0; i <= last - first; ++i)
    for (long k = 0; k < nd; ++k) {
      double r;
      if (!to_real(c[(size_t)(i * nd + k)], r)) return 7;
      m.x[3 * (size_t)(first - 1 + i) + (size_t)k] = r;
    }
  skip_record(T);
  return 0;
}

int sec_cells(Tokens& T, MgpuCasMesh& m) {
  std::vector<std::string> h;
  if (!read_group(T, h)) {
    skip_record(T);
    return 0;
  }
  if (h.size() < 4) return 8;
  long v[4];
  for (int k = 0; k < 4; ++k)
    if (!to_int(h[(size_t)k], v[k])) {  // named definition record
      skip_record(T);
      return 0;
    }
  if (v[0] != 0 && v[2] > m.ncells) m.ncells = (int32_t)v[2];
  skip_record(T);
  return 0;
}

int sec_faces(Tokens& T, std::vector<FaceRec>& faces, int32_t& nfaces) {
  std::vector<std::string> h, g;
  if (!read_group(T, h) || h.size() < 4) return 9;
  long v[5] = {0, 0, 0, 0, 0};
  for (size_t k = 0; k < h.size() && k < 4; ++k)
    if (!to_int(h[k], v[k])) {  // a name field: definition record
      skip_record(T);
      return 0;
    }
  const long zid = v[0], first = v[1], last = v[2], cond = v[3];
  if (zid == 0 || cond == 0 || h.size() == 4 || !to_int(h[4], v[4])) {  // declaration / definition
    skip_record(T);
    return 0;
  }
  const long ftype = v[4];
  if (first < 1 || last < first) return 10;
  if (!read_group(T, g)) return 10;
  if ((long)faces.size() < last) faces.resize((size_t)last);
  size_t p = 0;
  auto next = [&](long& out) -> bool { return p < g.size() && to_int(g[p++], out); };
  for (long k = first; k <= last; ++k) {
    long ft = ftype, nn = 0;
    if (ftype == 0 && !next(ft)) return 10;
    if (ft == 2 || ft == 3 || ft == 4) {
      nn = ft;
    } else if (ft == 5) {
      if (!next(nn) || nn < 1) return 10;
    } else {
      return 11;  // unknown face type
    }
    FaceRec& f = faces[(size_t)(k - 1)];
    f.nodes.resize((size_t)nn);
    for (long j = 0; j < nn; ++j) {
      long nd;
      if (!next(nd)) return 10;
      f.nodes[(size_t)j] = (int32_t)nd;
    }
    long a, b;
    if (!next(a) || !next(b)) return 10;
    f.c0 = (int32_t)a;
    f.c1 = (int32_t)b;
    f.zone = (int32_t)zid;
    f.set = true;
  }
  if (last > nfaces) nfaces = (int32_t)last;
  skip_record(T);
  return 0;
}

void sec_zonedef(Tokens& T, MgpuCasMesh& m) {
  std::vector<std::string> h;
  if (read_group(T, h) && h.size() >= 2) {
    long id;
    if (to_int(h[0], id)) m.zone_names[(int)id] = h[1];
  }
  skip_record(T);
}

}  // namespace

extern "C" {

int mgpu_cas_read(const char* path, MgpuMesh* mesh, MgpuCasMesh** holder, int* ier) {
  if (!path || !mesh || !holder || !ier) return MGPU_E_ARG;
  *holder = nullptr;
  *ier = 0;
  FILE* fp = std::fopen(path, "rb");
  if (!fp) {
    *ier = 1;
    return 0;
  }
  std::string text;
  char buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof(buf), fp)) > 0) text.append(buf, got);
  std::fclose(fp);

  MgpuCasMesh* m = new MgpuCasMesh();
  Tokens T;
  tokenize(text, T.t);
  text.clear();
  std::vector<FaceRec> faces;
  int32_t nfaces = 0;
  int e = 0;
  while (!T.end() && !e) {
    if (T.t[T.p++] != "(") continue;
    if (T.end()) break;
    const std::string sec = T.t[T.p++];
    if (sec == "10") e = sec_nodes(T, *m);
    else if (sec == "12") e = sec_cells(T, *m);
    else if (sec == "13") e = sec_faces(T, faces, nfaces);
    else if (sec == "45") sec_zonedef(T, *m);
    else skip_record(T);
  }
  if (!e && (m->nnodes == 0 || m->ncells == 0 || nfaces == 0)) e = 20;  // incomplete mesh
  if (!e) {
    m->nfaces = nfaces;
    m->fnode_ptr.assign(1, 0);
    for (int32_t k = 0; k < nfaces && !e; ++k) {
      const FaceRec& f = faces[(size_t)k];
      if (!f.set) {
        e = 20;  // a face index no record covered
        break;
      }
      for (int32_t nd : f.nodes) {
        if (nd < 1 || nd > m->nnodes) e = 21;
        m->fnodes.push_back(nd);
      }
      if (f.c0 < 1 || f.c0 > m->ncells || f.c1 < 0 || f.c1 > m->ncells) e = 21;
      m->fnode_ptr.push_back((int32_t)m->fnodes.size());
      m->c0.push_back(f.c0);
      m->c1.push_back(f.c1);
      m->zone.push_back(f.zone);
    }
  }
  if (e) {
    delete m;
    *ier = e;
    return 0;
  }
  for (const auto& kv : m->zone_names) m->names_text += std::to_string(kv.first) + " " + kv.second + "\n";
  std::memset(mesh, 0, sizeof(*mesh));
  mesh->nnodes = m->nnodes;
  mesh->nfaces = m->nfaces;
  mesh->ncells = m->ncells;
  mesh->x = m->x.data();
  mesh->fnode_ptr = m->fnode_ptr.data();
  mesh->fnodes = m->fnodes.data();
  mesh->c0 = m->c0.data();
  mesh->c1 = m->c1.data();
  mesh->zone = m->zone.data();
  *holder = m;
  return 0;
}

int mgpu_cas_zone_names(const MgpuCasMesh* holder, char* buf, int cap, int* len) {
  if (!holder || !len) return MGPU_E_ARG;
  const std::string& s = holder->names_text;
  *len = (int)s.size();
  if (buf && cap > 0) {
    const int n = std::min<int>(cap - 1, (int)s.size());
    std::memcpy(buf, s.data(), (size_t)n);
    buf[n] = '\0';
  }
  return 0;
}

int mgpu_cas_free(MgpuCasMesh* holder) {
  delete holder;
  return 0;
}

}  // extern "C"
