// Host-side pieces of the C ABI that need no GPU: configuration (XML and
// command line), triangle meshes (.raw reader, icosphere, capsule) and the
// uniform geometry grid.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "dsmc_b200.h"
#include "dsmc_host.hpp"

namespace dsmcb {

// ------------------------------------------------------------------ XML ----
// A small XML reader for the configuration files: elements, attributes, text,
// comments and the <?xml?> prolog.  Entities are not expanded.

namespace {

struct XNode {
  std::string name;
  std::map<std::string, std::string> attr;
  std::string text;
  std::vector<std::unique_ptr<XNode>> kids;
  const XNode* child(const char* n) const {
    for (auto& k : kids)
      if (k->name == n) return k.get();
    return nullptr;
  }
};

struct XParser {
  const std::string& s;
  size_t i = 0;
  bool ok = true;
  explicit XParser(const std::string& src) : s(src) {}
  void ws() { while (i < s.size() && isspace((unsigned char)s[i])) i++; }
  bool starts(const char* p) const { return s.compare(i, strlen(p), p) == 0; }
  void skip_misc() {
    for (;;) {
      ws();
      if (starts("<?")) {
        size_t e = s.find("?>", i);
        i = e == std::string::npos ? s.size() : e + 2;
      } else if (starts("<!--")) {
        size_t e = s.find("-->", i);
        i = e == std::string::npos ? s.size() : e + 3;
      } else if (starts("<!")) {
        size_t e = s.find('>', i);
        i = e == std::string::npos ? s.size() : e + 1;
      } else {
        return;
      }
    }
  }
  std::string name() {
    size_t b = i;
    while (i < s.size() && (isalnum((unsigned char)s[i]) || s[i] == '_' || s[i] == '-' ||
                            s[i] == ':' || s[i] == '.'))
      i++;
    return s.substr(b, i - b);
  }
  std::unique_ptr<XNode> element() {
    skip_misc();
    if (i >= s.size() || s[i] != '<') { ok = false; return nullptr; }
    i++;
    auto n = std::make_unique<XNode>();
    n->name = name();
    if (n->name.empty()) { ok = false; return nullptr; }
    for (;;) {
      ws();
      if (i >= s.size()) { ok = false; return nullptr; }
      if (s[i] == '/') {
        if (i + 1 < s.size() && s[i + 1] == '>') { i += 2; return n; }
        ok = false; return nullptr;
      }
      if (s[i] == '>') { i++; break; }
      std::string an = name();
      if (an.empty()) { ok = false; return nullptr; }
      ws();
      if (i >= s.size() || s[i] != '=') { ok = false; return nullptr; }
      i++;
      ws();
      if (i >= s.size() || (s[i] != '"' && s[i] != '\'')) { ok = false; return nullptr; }
      char q = s[i++];
      size_t e = s.find(q, i);
      if (e == std::string::npos) { ok = false; return nullptr; }
      n->attr[an] = s.substr(i, e - i);
      i = e + 1;
    }
    for (;;) {
      if (i >= s.size()) { ok = false; return nullptr; }
      if (starts("<!--")) {
        size_t e = s.find("-->", i);
        i = e == std::string::npos ? s.size() : e + 3;
        continue;
      }
      if (starts("</")) {
        i += 2;
        std::string en = name();
        ws();
        if (en != n->name || i >= s.size() || s[i] != '>') { ok = false; return nullptr; }
        i++;
        return n;
      }
      if (s[i] == '<') {
        auto k = element();
        if (!k) return nullptr;
        n->kids.push_back(std::move(k));
        continue;
      }
      n->text.push_back(s[i++]);
    }
  }
};

bool read_file(const std::string& path, std::string& out) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  std::stringstream ss;
  ss << f.rdbuf();
  out = ss.str();
  return true;
}

std::unique_ptr<XNode> parse_xml(const std::string& text) {
  XParser p(text);
  auto root = p.element();
  if (!p.ok) return nullptr;
  return root;
}

int face_index(const std::string& side) {
  static const char* names[6] = {"-x", "+x", "-y", "+y", "-z", "+z"};
  for (int i = 0; i < 6; i++)
    if (side == names[i]) return i;
  return -1;
}

int face_kind_of(const std::string& k) {
  if (k == "specular" || k == "wall") return DSMC_FACE_SPECULAR;
  if (k == "diffuse") return DSMC_FACE_DIFFUSE;
  if (k == "outflow") return DSMC_FACE_OUTFLOW;
  if (k == "periodic") return DSMC_FACE_PERIODIC;
  if (k == "inflow") return DSMC_FACE_INFLOW;
  return -1;
}

}  // namespace

std::string g_config_error;

int config_default(dsmc_config* c) {
  std::memset(c, 0, sizeof(*c));
  // settings_t::settings_t, src/sim_settings.cpp:35-44, include/dsmc.h
  c->grid_min[0] = 0.0f; c->grid_min[1] = 0.0f; c->grid_min[2] = 0.0f;
  c->grid_max[0] = 0.3f; c->grid_max[1] = 0.18f; c->grid_max[2] = 0.18f;
  c->grid_dim[0] = 30; c->grid_dim[1] = 18; c->grid_dim[2] = 18;
  c->density = 1.0e20f;
  c->fnum = 0.2e14f;
  c->temp = 300.0f;
  c->periodic = 'n';
  c->gas_mass = 5.0e-26f;
  c->gas_diam = 3.5e-10f;
  c->gas_tref = 273.0f;
  c->dt = 2e-6f;
  c->geometry = 0;
  c->benchmark = 1;
  c->gas_omega = 0.5f;
  c->ntc_local = 0;
  c->rng = DSMC_RNG_TAUS;
  c->seed = 999;  // SEED, include/MersenneTwister.h:17
  c->face_mode = 0;
  for (int i = 0; i < 6; i++) { c->face_kind[i] = DSMC_FACE_SPECULAR; c->face_temp[i] = 300.f; }
  c->wall_diffuse = 0;
  c->wall_temp = 300.f;
  c->init_kind = DSMC_INIT_REFERENCE;
  c->init_temp2 = 0.f;
  c->sample_every = 100;
  c->capacity_factor = 1.0f;
  c->part_per_cell = 0;
  return DSMC_OK;
}

static bool scan3f(const XNode* n, float* v) {
  return n && std::sscanf(n->text.c_str(), "%f %f %f", &v[0], &v[1], &v[2]) == 3;
}

int config_read_xml(const char* path, dsmc_config* c) {
  std::string text;
  if (!read_file(path, text)) {
    g_config_error = std::string("cannot read ") + path;
    return DSMC_ERR_IO;
  }
  auto root = parse_xml(text);
  if (!root) {
    g_config_error = std::string("malformed XML in ") + path;
    return DSMC_ERR_CONFIG;
  }
  const XNode* grid = root->child("grid");
  if (!grid || !scan3f(grid->child("min"), c->grid_min) || !scan3f(grid->child("max"), c->grid_max) ||
      !grid->child("dim") ||
      std::sscanf(grid->child("dim")->text.c_str(), "%d %d %d", &c->grid_dim[0], &c->grid_dim[1],
                  &c->grid_dim[2]) != 3) {
    g_config_error = "missing or malformed <grid><min/max/dim>";
    return DSMC_ERR_CONFIG;
  }
  auto f1 = [&](const char* tag, float* v) -> bool {
    const XNode* n = root->child(tag);
    if (!n) return false;
    return std::sscanf(n->text.c_str(), "%f", v) == 1;
  };
  if (!f1("density", &c->density) || !f1("fnum", &c->fnum) || !f1("temp", &c->temp)) {
    g_config_error = "missing <density>, <fnum> or <temp>";
    return DSMC_ERR_CONFIG;
  }
  if (const XNode* sv = root->child("streamvel")) scan3f(sv, c->stream_vel);
  if (const XNode* pc = root->child("periodic")) {
    size_t k = pc->text.find_first_not_of(" \t\r\n");
    if (k != std::string::npos) c->periodic = pc->text[k];
  }
  f1("dt", &c->dt);
  // extension tags
  f1("omega", &c->gas_omega);
  if (const XNode* w = root->child("wall")) {
    auto it = w->attr.find("kind");
    if (it != w->attr.end()) c->wall_diffuse = it->second == "diffuse";
    it = w->attr.find("T");
    if (it == w->attr.end()) it = w->attr.find("temp");
    if (it != w->attr.end()) c->wall_temp = (float)std::atof(it->second.c_str());
    it = w->attr.find("hit");
    if (it != w->attr.end()) c->geom_nearest = it->second == "nearest";
  }
  for (auto& k : root->kids) {
    if (k->name != "face") continue;
    auto s = k->attr.find("side");
    auto kd = k->attr.find("kind");
    if (s == k->attr.end() || kd == k->attr.end()) {
      g_config_error = "<face> needs side= and kind=";
      return DSMC_ERR_CONFIG;
    }
    int fi = face_index(s->second), fk = face_kind_of(kd->second);
    if (fi < 0 || fk < 0) {
      g_config_error = "bad <face side/kind>: " + s->second + " " + kd->second;
      return DSMC_ERR_CONFIG;
    }
    c->face_mode = 1;
    c->face_kind[fi] = fk;
    auto t = k->attr.find("T");
    if (t != k->attr.end()) c->face_temp[fi] = (float)std::atof(t->second.c_str());
  }
  if (const XNode* r = root->child("rng")) {
    if (r->text.find("philox") != std::string::npos) c->rng = DSMC_RNG_PHILOX;
    else if (r->text.find("taus") != std::string::npos) c->rng = DSMC_RNG_TAUS;
  }
  if (const XNode* sd = root->child("seed")) c->seed = std::strtoull(sd->text.c_str(), nullptr, 10);
  if (const XNode* sm = root->child("sample")) {
    auto it = sm->attr.find("every");
    if (it != sm->attr.end()) c->sample_every = std::atoi(it->second.c_str());
  }
  if (const XNode* nt = root->child("ntc")) c->ntc_local = nt->text.find("local") != std::string::npos;
  if (const XNode* in = root->child("init")) {
    auto it = in->attr.find("kind");
    if (it != in->attr.end()) {
      if (it->second == "maxwell") c->init_kind = DSMC_INIT_MAXWELL;
      else if (it->second == "bimodal") c->init_kind = DSMC_INIT_BIMODAL;
      else c->init_kind = DSMC_INIT_REFERENCE;
    }
    it = in->attr.find("T2");
    if (it != in->attr.end()) c->init_temp2 = (float)std::atof(it->second.c_str());
  }
  // gas
  const XNode* gas = root->child("gas");
  if (!gas || gas->attr.find("file") == gas->attr.end()) {
    g_config_error = "missing <gas file=...>";
    return DSMC_ERR_CONFIG;
  }
  std::string gas_file = gas->attr.at("file");
  std::string gas_name = gas->text;
  size_t a = gas_name.find_first_not_of(" \t\r\n"), b = gas_name.find_last_not_of(" \t\r\n");
  gas_name = a == std::string::npos ? "" : gas_name.substr(a, b - a + 1);
  std::string gtext;
  if (!read_file(gas_file, gtext)) {
    // the reference opens it relative to the working directory (its own root);
    // also try the config's directory and that directory's parent
    std::string dir = path;
    size_t sl = dir.find_last_of('/');
    dir = sl == std::string::npos ? "./" : dir.substr(0, sl + 1);
    if (!read_file(dir + gas_file, gtext) && !read_file(dir + "../" + gas_file, gtext)) {
      g_config_error = "cannot read gas file " + gas_file;
      return DSMC_ERR_IO;
    }
  }
  auto groot = parse_xml(gtext);
  if (!groot) {
    g_config_error = "malformed gas file " + gas_file;
    return DSMC_ERR_CONFIG;
  }
  const XNode* g = nullptr;
  for (auto& k : groot->kids) {
    auto it = k->attr.find("name");
    if (k->name == "gas" && it != k->attr.end() && it->second == gas_name) g = k.get();
  }
  if (!g) {
    g_config_error = "gas '" + gas_name + "' not in " + gas_file;
    return DSMC_ERR_CONFIG;
  }
  auto gf = [&](const char* tag, float* v) {
    const XNode* n = g->child(tag);
    if (n) std::sscanf(n->text.c_str(), "%f", v);
  };
  gf("mass", &c->gas_mass);
  gf("diam", &c->gas_diam);
  gf("temp", &c->gas_tref);
  gf("omega", &c->gas_omega);
  return DSMC_OK;
}

int config_from_args(int argc, const char* const* argv, dsmc_config* c, float* run_for) {
  if (run_for) *run_for = -1.0f;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    auto need = [&](void) -> const char* {
      if (i + 1 >= argc) return nullptr;
      return argv[++i];
    };
    if (a == "-f") {
      const char* p = need();
      if (!p) { g_config_error = "-f needs a file"; return DSMC_ERR_ARG; }
      int st = config_read_xml(p, c);
      if (st) return st;
    } else if (a == "-benchmark") {
      c->benchmark = 1;
    } else if (a == "-cpu") {
      // parsed and ignored, as in the reference (src/sim_settings.cpp:150-154)
    } else if (a == "-no-geometry") {
      c->geometry = 0;
    } else if (a == "-geometry") {
      c->geometry = 1;
    } else if (a == "-mt") {
      g_config_error = "-mt (Mersenne-Twister collisions) is not supported; use the default HybridTaus";
      return DSMC_ERR_ARG;
    } else if (a == "-density") {
      const char* p = need();
      if (!p) return DSMC_ERR_ARG;
      c->density = (float)std::atof(p);
    } else if (a == "-dt") {
      const char* p = need();
      if (!p) return DSMC_ERR_ARG;
      c->dt = (float)std::atof(p);
    } else if (a == "-run-for") {
      const char* p = need();
      if (!p) return DSMC_ERR_ARG;
      if (run_for) *run_for = (float)std::atof(p);
    }
  }
  return DSMC_OK;
}

// ----------------------------------------------------------------- mesh ----

int read_raw_mesh(const char* path, std::vector<float>& verts, std::vector<uint32_t>& tris,
                  std::vector<float>& fnorm) {
  // Model::LoadRaw, src/model.cpp:348-401: "RW", two version ints, bbox
  // (6 floats), then u32-counted arrays: vertices (vec3), texCoords (vec2),
  // normals (vec3), facesNorm (vec3), colors (vec3), indices (u32).  The grid
  // section that follows is not needed (the grid is rebuilt).
  std::ifstream f(path, std::ios::binary);
  if (!f) return DSMC_ERR_IO;
  char mg[2];
  f.read(mg, 2);
  if (!f || mg[0] != 'R' || mg[1] != 'W') return DSMC_ERR_IO;
  int32_t ver[2];
  float bbox[6];
  f.read((char*)ver, sizeof(ver));
  f.read((char*)bbox, sizeof(bbox));
  auto arr = [&](size_t esz, std::vector<char>& out) -> bool {
    uint32_t n = 0;
    f.read((char*)&n, 4);
    if (!f) return false;
    out.resize((size_t)n * esz);
    if (n) f.read(out.data(), out.size());
    return (bool)f;
  };
  std::vector<char> v, tex, nrm, fn, col, idx;
  if (!arr(12, v) || !arr(8, tex) || !arr(12, nrm) || !arr(12, fn) || !arr(12, col) || !arr(4, idx))
    return DSMC_ERR_IO;
  verts.resize(v.size() / 4);
  std::memcpy(verts.data(), v.data(), v.size());
  tris.resize(idx.size() / 4);
  std::memcpy(tris.data(), idx.data(), idx.size());
  fnorm.resize(fn.size() / 4);
  std::memcpy(fnorm.data(), fn.data(), fn.size());
  if (tris.size() % 3) return DSMC_ERR_IO;
  for (uint32_t t : tris)
    if ((size_t)t * 3 >= verts.size()) return DSMC_ERR_IO;
  return DSMC_OK;
}

void face_normals(const std::vector<float>& v, const std::vector<uint32_t>& t, std::vector<float>& n) {
  // calc_normal (src/vector.cpp:72-75): norm(cross(v2 - v1, v3 - v1))
  size_t nt = t.size() / 3;
  n.resize(nt * 3);
  for (size_t i = 0; i < nt; i++) {
    const float* a = &v[3 * (size_t)t[3 * i]];
    const float* b = &v[3 * (size_t)t[3 * i + 1]];
    const float* c = &v[3 * (size_t)t[3 * i + 2]];
    float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    float e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    float x = e1[1] * e2[2] - e1[2] * e2[1];
    float y = e1[2] * e2[0] - e1[0] * e2[2];
    float z = e1[0] * e2[1] - e1[1] * e2[0];
    float l = std::sqrt(x * x + y * y + z * z);
    if (l > 0) { x /= l; y /= l; z /= l; }
    n[3 * i] = x; n[3 * i + 1] = y; n[3 * i + 2] = z;
  }
}

void mesh_icosphere(int level, float radius, const float* center, std::vector<float>& verts,
                    std::vector<uint32_t>& tris) {
  const double t = (1.0 + std::sqrt(5.0)) / 2.0;
  std::vector<double> p = {-1, t, 0, 1, t, 0, -1, -t, 0, 1, -t, 0, 0, -1, t, 0, 1, t,
                           0, -1, -t, 0, 1, -t, t, 0, -1, t, 0, 1, -t, 0, -1, -t, 0, 1};
  for (size_t i = 0; i < p.size(); i += 3) {
    double l = std::sqrt(p[i] * p[i] + p[i + 1] * p[i + 1] + p[i + 2] * p[i + 2]);
    p[i] /= l; p[i + 1] /= l; p[i + 2] /= l;
  }
  std::vector<uint32_t> f = {0, 11, 5, 0, 5, 1,  0, 1, 7,  0, 7, 10, 0, 10, 11,
                             1, 5, 9, 5, 11, 4, 11, 10, 2, 10, 7, 6, 7, 1, 8,
                             3, 9, 4, 3, 4, 2,  3, 2, 6,  3, 6, 8,  3, 8, 9,
                             4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7,  9, 8, 1};
  for (int lv = 0; lv < level; lv++) {
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> mid;
    auto midpoint = [&](uint32_t a, uint32_t b) {
      auto key = std::make_pair(std::min(a, b), std::max(a, b));
      auto it = mid.find(key);
      if (it != mid.end()) return it->second;
      double x = p[3 * a] + p[3 * b], y = p[3 * a + 1] + p[3 * b + 1], z = p[3 * a + 2] + p[3 * b + 2];
      double l = std::sqrt(x * x + y * y + z * z);
      uint32_t id = (uint32_t)(p.size() / 3);
      p.push_back(x / l); p.push_back(y / l); p.push_back(z / l);
      mid[key] = id;
      return id;
    };
    std::vector<uint32_t> g;
    for (size_t i = 0; i < f.size(); i += 3) {
      uint32_t a = f[i], b = f[i + 1], c = f[i + 2];
      uint32_t ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
      uint32_t nt[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
      g.insert(g.end(), nt, nt + 12);
    }
    f.swap(g);
  }
  verts.resize(p.size());
  for (size_t i = 0; i < p.size(); i += 3) {
    verts[i] = (float)(center[0] + radius * p[i]);
    verts[i + 1] = (float)(center[1] + radius * p[i + 1]);
    verts[i + 2] = (float)(center[2] + radius * p[i + 2]);
  }
  tris = f;
}

// Sphere-cone capsule around the +x axis: spherical nose of radius rn facing
// -x, a cone of half-angle theta tangent to it, a flat base closing the body
// at total length `length` from the nose tip.  Rings along the profile are
// about one edge length h apart and each ring has about 2 pi r / h vertices,
// so the triangles are near-equilateral of similar size everywhere (no fan of
// slivers at the nose tip or the base centre); h is chosen for about
// ntarget triangles.  The seed rotates the azimuthal start of the rings.
void mesh_capsule(float rn, float theta_deg, float length, const float* c, uint32_t ntarget,
                  uint64_t seed, std::vector<float>& verts, std::vector<uint32_t>& tris) {
  const double th = theta_deg * M_PI / 180.0;
  const double phi_t = M_PI / 2 - th;  // polar angle of the tangency from the nose axis
  const double x_tip = c[0] - rn;
  const double x_t = c[0] - rn * std::cos(phi_t), r_t = rn * std::sin(phi_t);
  const double x_base = x_tip + length;
  const double r_base = r_t + (x_base - x_t) * std::tan(th);
  const double L1 = rn * phi_t;
  const double L2 = std::hypot(x_base - x_t, r_base - r_t);
  const double L3 = r_base;
  const double area = 2 * M_PI * rn * rn * (1 - std::cos(phi_t)) + M_PI * (r_t + r_base) * L2 +
                      M_PI * r_base * r_base;
  const double h = std::sqrt(4.0 * area / (std::sqrt(3.0) * std::max<uint32_t>(ntarget, 64)));
  const double ds = h * std::sqrt(3.0) / 2;  // ring spacing along the profile
  const uint32_t n1 = std::max<uint32_t>(2, (uint32_t)std::lround(L1 / ds));
  const uint32_t n2 = std::max<uint32_t>(1, (uint32_t)std::lround(L2 / ds));
  const uint32_t n3 = std::max<uint32_t>(2, (uint32_t)std::lround(L3 / ds));
  // splitmix64 of the seed -> azimuthal phase
  uint64_t z = seed + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  const double phase = (double)(z >> 11) / 9007199254740992.0 * 2 * M_PI;
  std::vector<double> rx, rr;  // profile rings (x, radius), excluding the two poles
  for (uint32_t i = 1; i <= n1; i++) {
    const double ph = phi_t * i / n1;
    rx.push_back(c[0] - rn * std::cos(ph));
    rr.push_back(rn * std::sin(ph));
  }
  for (uint32_t i = 1; i <= n2; i++) {
    const double x = x_t + (x_base - x_t) * i / n2;
    rx.push_back(x);
    rr.push_back(r_t + (x - x_t) * std::tan(th));
  }
  for (uint32_t i = 1; i < n3; i++) {
    rx.push_back(x_base);
    rr.push_back(r_base * (1.0 - (double)i / n3));
  }
  verts.clear();
  tris.clear();
  auto push = [&](double x, double y, double zz) {
    verts.push_back((float)x); verts.push_back((float)y); verts.push_back((float)zz);
    return (uint32_t)(verts.size() / 3 - 1);
  };
  const uint32_t tip = push(x_tip, c[1], c[2]);
  std::vector<uint32_t> first(rx.size()), count(rx.size());
  for (size_t k = 0; k < rx.size(); k++) {
    const uint32_t m = std::max<uint32_t>(3, (uint32_t)std::lround(2 * M_PI * rr[k] / h));
    first[k] = (uint32_t)(verts.size() / 3);
    count[k] = m;
    for (uint32_t a = 0; a < m; a++) {
      const double ang = phase + 2 * M_PI * a / m;
      push(rx[k], c[1] + rr[k] * std::cos(ang), c[2] + rr[k] * std::sin(ang));
    }
  }
  const uint32_t tail = push(x_base, c[1], c[2]);
  auto rid = [&](size_t k, uint32_t a) { return first[k] + a % count[k]; };
  // outward winding: looking from outside, counter-clockwise
  for (uint32_t a = 0; a < count[0]; a++) {
    tris.push_back(tip); tris.push_back(rid(0, a + 1)); tris.push_back(rid(0, a));
  }
  // band between ring k and k+1: advance along whichever ring's next vertex
  // comes first in angle (all rings start at the same phase)
  for (size_t k = 0; k + 1 < rx.size(); k++) {
    const uint32_t ma = count[k], mb = count[k + 1];
    uint32_t i = 0, j = 0;
    while (i < ma || j < mb) {
      const bool step_a = j == mb || (i < ma && (double)(i + 1) / ma < (double)(j + 1) / mb);
      if (step_a) {
        tris.push_back(rid(k, i)); tris.push_back(rid(k, i + 1)); tris.push_back(rid(k + 1, j));
        i++;
      } else {
        tris.push_back(rid(k, i)); tris.push_back(rid(k + 1, j + 1)); tris.push_back(rid(k + 1, j));
        j++;
      }
    }
  }
  const size_t last = rx.size() - 1;
  for (uint32_t a = 0; a < count[last]; a++) {
    tris.push_back(tail); tris.push_back(rid(last, a)); tris.push_back(rid(last, a + 1));
  }
}

// ----------------------------------------------------------------- grid ----

// Separating-axis triangle/box test (Akenine-Moller, "Fast 3D Triangle-Box
// Overlap Testing", 2001): disjoint iff the projections are disjoint on one of
// 13 axes (3 box normals, the triangle normal, 9 edge x box-normal crosses).
bool tri_box_overlap(const float center[3], const float half[3], const float tri[9]) {
  float v[3][3];
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++) v[i][k] = tri[3 * i + k] - center[k];
  float e[3][3];
  for (int k = 0; k < 3; k++) {
    e[0][k] = v[1][k] - v[0][k];
    e[1][k] = v[2][k] - v[1][k];
    e[2][k] = v[0][k] - v[2][k];
  }
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) {
      float a[3] = {0, 0, 0};
      if (j == 0) { a[1] = -e[i][2]; a[2] = e[i][1]; }
      if (j == 1) { a[0] = e[i][2]; a[2] = -e[i][0]; }
      if (j == 2) { a[0] = -e[i][1]; a[1] = e[i][0]; }
      float p0 = a[0] * v[0][0] + a[1] * v[0][1] + a[2] * v[0][2];
      float p1 = a[0] * v[1][0] + a[1] * v[1][1] + a[2] * v[1][2];
      float p2 = a[0] * v[2][0] + a[1] * v[2][1] + a[2] * v[2][2];
      float mn = std::min(std::min(p0, p1), p2);
      float mx = std::max(std::max(p0, p1), p2);
      float r = half[0] * std::fabs(a[0]) + half[1] * std::fabs(a[1]) + half[2] * std::fabs(a[2]);
      if (mn > r || mx < -r) return false;
    }
  }
  for (int k = 0; k < 3; k++) {
    float mn = std::min(std::min(v[0][k], v[1][k]), v[2][k]);
    float mx = std::max(std::max(v[0][k], v[1][k]), v[2][k]);
    if (mn > half[k] || mx < -half[k]) return false;
  }
  float n[3] = {e[0][1] * e[1][2] - e[0][2] * e[1][1], e[0][2] * e[1][0] - e[0][0] * e[1][2],
                e[0][0] * e[1][1] - e[0][1] * e[1][0]};
  float d = n[0] * v[0][0] + n[1] * v[0][1] + n[2] * v[0][2];
  float r = half[0] * std::fabs(n[0]) + half[1] * std::fabs(n[1]) + half[2] * std::fabs(n[2]);
  return !(d > r || d < -r);
}

// Model::CreateGrid + reg_grid_t::encloseGrid (src/model.cpp:733-769,
// src/reggrid.cpp:27-93).  Each triangle is tested against the cells its
// bounding box touches (plus one cell of margin); entries stay in triangle
// order within a cell, the order the reference's cell-major loop produces.
void geometry_grid_frame(const float* verts, uint32_t nverts, const int dim[3], GeomGrid& out) {
  float mn[3] = {100000, 100000, 100000}, mx[3] = {-100000, -100000, -100000};
  for (uint32_t i = 0; i < nverts; i++)
    for (int k = 0; k < 3; k++) {
      float x = verts[3 * (size_t)i + k];
      if (x < mn[k]) mn[k] = x;
      if (x > mx[k]) mx[k] = x;
    }
  for (int k = 0; k < 3; k++) {
    out.dim[k] = (uint32_t)dim[k];
    out.cell[k] = (mx[k] - mn[k]) / (float)(uint32_t)dim[k];
    out.bbox[k] = mn[k];
    out.bbox[3 + k] = mx[k];
  }
}

void build_geometry_grid(const float* verts, uint32_t nverts, const uint32_t* tris, uint32_t ntris,
                         const int dim[3], GeomGrid& out) {
  geometry_grid_frame(verts, nverts, dim, out);
  const float mn[3] = {out.bbox[0], out.bbox[1], out.bbox[2]};
  const uint32_t dx = out.dim[0], dy = out.dim[1], dz = out.dim[2];
  const uint32_t ncell = dx * dy * dz;
  std::vector<std::vector<uint32_t>> bins(ncell);
  out.flags.assign(ncell, 0);
  for (uint32_t t = 0; t < ntris; t++) {
    float tri[9];
    float tmn[3] = {1e30f, 1e30f, 1e30f}, tmx[3] = {-1e30f, -1e30f, -1e30f};
    for (int q = 0; q < 3; q++)
      for (int k = 0; k < 3; k++) {
        float x = verts[3 * (size_t)tris[3 * t + q] + k];
        tri[3 * q + k] = x;
        tmn[k] = std::min(tmn[k], x);
        tmx[k] = std::max(tmx[k], x);
      }
    int lo[3], hi[3];
    for (int k = 0; k < 3; k++) {
      double a = std::floor((tmn[k] - mn[k]) / out.cell[k]) - 1;
      double b = std::floor((tmx[k] - mn[k]) / out.cell[k]) + 1;
      lo[k] = (int)std::max(0.0, a);
      hi[k] = (int)std::min((double)out.dim[k] - 1, b);
    }
    for (int z = lo[2]; z <= hi[2]; z++)
      for (int y = lo[1]; y <= hi[1]; y++)
        for (int x = lo[0]; x <= hi[0]; x++) {
          float bmin[3] = {mn[0] + (float)(uint32_t)x * out.cell[0],
                           mn[1] + (float)(uint32_t)y * out.cell[1],
                           mn[2] + (float)(uint32_t)z * out.cell[2]};
          float center[3], half[3];
          for (int k = 0; k < 3; k++) {
            float bmax = bmin[k] + out.cell[k];
            half[k] = (bmax - bmin[k]) / 2;
            center[k] = bmin[k] + half[k];
          }
          if (tri_box_overlap(center, half, tri)) {
            uint32_t c = dx * dy * (uint32_t)z + dx * (uint32_t)y + (uint32_t)x;
            bins[c].push_back(t);
            out.flags[c] = 1;
          }
        }
  }
  // enclose: along z, cells between a flagged cell and the next flagged cell
  // become flagged (src/reggrid.cpp:49-79)
  for (uint32_t x = 0; x < dx; x++)
    for (uint32_t y = 0; y < dy; y++) {
      bool last_full = false;
      uint32_t last_z = 0;
      for (uint32_t z = 0; z < dz; z++) {
        if (out.flags[dx * dy * z + dx * y + x]) {
          if (!last_full) {
            last_z = z;
            last_full = true;
          } else {
            while (last_z != z) {
              out.flags[dx * dy * last_z + dx * y + x] = 1;
              last_z++;
            }
            last_full = false;
          }
        }
      }
    }
  out.count.resize(ncell);
  out.tri_ids.clear();
  for (uint32_t c = 0; c < ncell; c++) {
    out.count[c] = (uint32_t)bins[c].size();
    out.tri_ids.insert(out.tri_ids.end(), bins[c].begin(), bins[c].end());
  }
}

}  // namespace dsmcb
