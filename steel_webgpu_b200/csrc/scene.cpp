// Scene files to the packed form on the host: scene.json reader and Sim.build (sim.js:95-521).
//
// The packer produces, word for word, the buffers the reference's Sim.build uploads: the static
// vec4 buffer statF (sim.js:212-233, 257-393), the u32 buffer statU with its collision-filter
// bitset (sim.js:234-255, 334-393), the compile-time constant table (sim.js:395-477) and the
// initial pose, velocity and articulation state (sim.js:478-502). Quantities the reference
// computes in JavaScript doubles (quatRotate, inv3, the hull bounding boxes, body radii) are
// computed in double here and rounded once to float, as a Float32Array store rounds them.
#include "scene.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>

namespace steel {
namespace scene {

// --- JSON -------------------------------------------------------------------------------------
static const JV kNull;

const JV* JV::get(const char* key) const {
  if (kind != Obj) return nullptr;
  for (const auto& kv : o)
    if (kv.first == key) return &kv.second;
  return nullptr;
}
bool JV::truthy() const {
  switch (kind) {
    case Null: return false;
    case Bool: return b;
    case Num: return n != 0.0;
    case Str: return !s.empty();
    case Arr: return !a.empty();
    case Obj: return !o.empty();
  }
  return false;
}
const JV& JV::operator[](size_t k) const { return (kind == Arr && k < a.size()) ? a[k] : kNull; }

namespace {

struct Reader {
  const char* p;
  const char* e;
  std::string err;
  void ws() {
    while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) p++;
  }
  bool lit(const char* w) {
    size_t n = std::strlen(w);
    if ((size_t)(e - p) < n || std::strncmp(p, w, n) != 0) return false;
    p += n;
    return true;
  }
  bool str(std::string& out) {
    if (p >= e || *p != '"') return false;
    p++;
    while (p < e && *p != '"') {
      char c = *p++;
      if (c == '\\') {
        if (p >= e) return false;
        char x = *p++;
        switch (x) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {
            if (e - p < 4) return false;
            unsigned v = (unsigned)std::strtoul(std::string(p, p + 4).c_str(), nullptr, 16);
            p += 4;
            if (v < 0x80) out += (char)v;
            else if (v < 0x800) { out += (char)(0xc0 | (v >> 6)); out += (char)(0x80 | (v & 0x3f)); }
            else { out += (char)(0xe0 | (v >> 12)); out += (char)(0x80 | ((v >> 6) & 0x3f)); out += (char)(0x80 | (v & 0x3f)); }
            break;
          }
          default: out += x;
        }
      } else {
        out += c;
      }
    }
    if (p >= e) return false;
    p++;
    return true;
  }
  bool value(JV& v, int depth) {
    if (depth > 64) { err = "JSON nested too deeply"; return false; }
    ws();
    if (p >= e) { err = "unexpected end of JSON"; return false; }
    char c = *p;
    if (c == '{') {
      p++;
      v.kind = JV::Obj;
      ws();
      if (p < e && *p == '}') { p++; return true; }
      for (;;) {
        ws();
        std::string k;
        if (!str(k)) { err = "expected a JSON key"; return false; }
        ws();
        if (p >= e || *p != ':') { err = "expected ':'"; return false; }
        p++;
        v.o.emplace_back(std::move(k), JV());
        if (!value(v.o.back().second, depth + 1)) return false;
        ws();
        if (p < e && *p == ',') { p++; continue; }
        if (p < e && *p == '}') { p++; return true; }
        err = "expected ',' or '}'";
        return false;
      }
    }
    if (c == '[') {
      p++;
      v.kind = JV::Arr;
      ws();
      if (p < e && *p == ']') { p++; return true; }
      for (;;) {
        v.a.emplace_back();
        if (!value(v.a.back(), depth + 1)) return false;
        ws();
        if (p < e && *p == ',') { p++; continue; }
        if (p < e && *p == ']') { p++; return true; }
        err = "expected ',' or ']'";
        return false;
      }
    }
    if (c == '"') {
      v.kind = JV::Str;
      if (!str(v.s)) { err = "bad JSON string"; return false; }
      return true;
    }
    if (lit("true")) { v.kind = JV::Bool; v.b = true; return true; }
    if (lit("false")) { v.kind = JV::Bool; v.b = false; return true; }
    if (lit("null")) { v.kind = JV::Null; return true; }
    if (lit("NaN")) { v.kind = JV::Num; v.n = NAN; return true; }
    if (lit("Infinity")) { v.kind = JV::Num; v.n = INFINITY; return true; }
    if (lit("-Infinity")) { v.kind = JV::Num; v.n = -INFINITY; return true; }
    // Number: strtod on a bounded copy (correctly rounded, like the reference's JSON.parse).
    const char* q = p;
    while (q < e && (std::strchr("+-0123456789.eE", *q) != nullptr)) q++;
    if (q == p) { err = std::string("unexpected character '") + c + "' in JSON"; return false; }
    std::string num(p, q);
    char* end = nullptr;
    v.kind = JV::Num;
    v.n = std::strtod(num.c_str(), &end);
    if (end != num.c_str() + num.size()) { err = "bad JSON number " + num; return false; }
    p = q;
    return true;
  }
};

}  // namespace

bool parse_json(const char* text, size_t len, JV& out, std::string& err) {
  Reader r{text, text + len, {}};
  out = JV();
  if (!r.value(out, 0)) { err = r.err.empty() ? "malformed JSON" : r.err; return false; }
  r.ws();
  if (r.p != r.e) { err = "trailing characters after JSON"; return false; }
  return true;
}

// --- packer -----------------------------------------------------------------------------------
namespace {

enum { JT_PRISMATIC = 0, JT_REVOLUTE = 1, JT_BALL = 2, JT_FIXED = 3, JT_FREE = 4, JT_DISTANCE = 5, JT_D6 = 6 };
constexpr uint32_t LB = 268;  // floats per link block (artwgsl.js:8)
constexpr int MAX_SUBSTEPS = 32;

struct Fail {
  std::string msg;
};
[[noreturn]] void fail(const std::string& m) { throw Fail{m}; }

const JV& need(const JV& o, const char* k) {
  const JV* v = o.get(k);
  if (!v) fail(std::string("scene.json: missing '") + k + "'");
  return *v;
}
// o.get(k) when present and not null, else nullptr (Python's `x.get(k) is not None`).
const JV* opt(const JV* o, const char* k) {
  if (!o) return nullptr;
  const JV* v = o->get(k);
  return (v && !v->is_null()) ? v : nullptr;
}
double num_or(const JV* o, const char* k, double def) {
  const JV* v = opt(o, k);
  return v ? v->num() : def;
}
// `x.get(k) or def`: def when missing, null, false, 0 or empty.
double num_or_falsy(const JV* o, const char* k, double def) {
  const JV* v = o ? o->get(k) : nullptr;
  return (v && v->truthy()) ? v->num() : def;
}
bool flag(const JV* o, const char* k) {
  const JV* v = o ? o->get(k) : nullptr;
  return v && v->truthy();
}
std::string str_or(const JV* o, const char* k, const std::string& def) {
  const JV* v = o ? o->get(k) : nullptr;
  return (v && v->truthy() && v->kind == JV::Str) ? v->s : def;
}

// sim.js:16-22, in double.
void quat_rotate(const double q[4], const double v[3], double r[3]) {
  const double x = q[0], y = q[1], z = q[2], w = q[3];
  const double ux = 2 * (x * v[0] + y * v[1] + z * v[2]);
  const double s2 = w * w - (x * x + y * y + z * z);
  const double cx = y * v[2] - z * v[1], cy = z * v[0] - x * v[2], cz = x * v[1] - y * v[0];
  r[0] = ux * x + s2 * v[0] + 2 * w * cx;
  r[1] = ux * y + s2 * v[1] + 2 * w * cy;
  r[2] = ux * z + s2 * v[2] + 2 * w * cz;
}
// sim.js:24-31, in double.
void inv3(const double m[9], double out[9]) {
  const double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
  const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
  const double det = a * A + b * B + c * C;
  if (std::fabs(det) < 1e-30) { for (int k = 0; k < 9; k++) out[k] = 0.0; return; }
  const double k = 1 / det;
  const double r[9] = {A * k, -(b * i - c * h) * k, (b * f - c * e) * k, B * k, (a * i - c * g) * k,
                       -(a * f - c * d) * k, C * k, -(a * h - b * g) * k, (a * e - b * d) * k};
  for (int t = 0; t < 9; t++) out[t] = r[t];
}
// Euclidean norm of three doubles, rounded once (extended-precision sum of squares).
double hypot3(double x, double y, double z) {
  long double s = (long double)x * x + (long double)y * y + (long double)z * z;
  return (double)std::sqrt(s);
}

struct Bin {
  const uint8_t* p;
  size_t n;
  // scene.bin view {off, n} as float32 / uint32 (LoadedScene.f32 / u32).
  template <class T> std::vector<T> view(const JV& r) const {
    const int64_t off = need(r, "off").i(), cnt = need(r, "n").i();
    if (off < 0 || cnt < 0 || (uint64_t)off + (uint64_t)cnt * sizeof(T) > n) fail("scene.bin range out of bounds");
    std::vector<T> out((size_t)cnt);
    if (cnt) std::memcpy(out.data(), p + off, (size_t)cnt * sizeof(T));
    return out;
  }
};

struct Dof {
  double armature, ke, kd, effort, lower, upper;
  int limited;
  uint32_t link;
  double damping, friction;
  double axis[3];
  bool scalar;
  double springKe, springRef, loadCoef, velLimit;
};
struct Link {
  int type, parent;
  uint32_t dof, ndof, nlin, qs, body, joint;
  bool movable;
};
struct Art { uint32_t linkStart, linkCount, dofStart, dofCount; };
struct Mimic { uint32_t art, f, l; double c0, c1; uint32_t fq, lq; };

// Python-style list element with a default when the list is missing, short or holds null.
double elem_or(const JV* list, size_t k, double def) {
  if (!list || list->kind != JV::Arr || k >= list->a.size() || list->a[k].is_null()) return def;
  return list->a[k].num();
}

std::string fmt_num(double v) {
  if (std::isfinite(v) && v == std::floor(v) && std::fabs(v) < 9.0e15) {
    char b[32];
    std::snprintf(b, sizeof b, "%lld", (long long)v);
    return b;
  }
  char b[40];
  std::snprintf(b, sizeof b, "%.17g", v);
  return b;
}

void pack_impl(const JV& S, const Bin& bin, const JV* o_in, Packed& P) {
  // Options (sim.js:63-84): scene defaults, then the caller's.
  const JV* Ssolver = opt(&S, "solver");
  double o_substeps = need(S, "substeps").num(), o_iterations = need(S, "iterations").num();
  double o_reg = Ssolver ? num_or_falsy(Ssolver, "contact_regularization", 0.0) : 0.0;
  if (!opt(Ssolver, "contact_regularization")) o_reg = 0.0;
  if (opt(o_in, "substeps")) o_substeps = opt(o_in, "substeps")->num();
  if (opt(o_in, "iterations")) o_iterations = opt(o_in, "iterations")->num();
  if (opt(o_in, "regularization")) o_reg = opt(o_in, "regularization")->num();
  const JV* o_solver = opt(o_in, "solver");
  if (o_substeps > MAX_SUBSTEPS) fail("at most 32 substeps");
  const JV& bodies = need(S, "bodies");
  const JV& J = need(S, "joints");
  const uint32_t NB = (uint32_t)need(bodies, "count").i();
  const JV* kin = opt(&bodies, "kinematic");
  auto is_kin = [&](uint32_t b) { return kin && b < kin->size() && (*kin)[b].truthy(); };
  const uint32_t NJ = (uint32_t)need(J, "count").i();
  const JV& jtype = need(J, "type");
  const JV& jchild = need(J, "child");
  const JV& jparent = need(J, "parent");
  const JV& jart = need(J, "articulation");
  const JV& q_start = need(J, "q_start");
  const JV& qd_start = need(J, "qd_start");
  const JV& jq = need(J, "q");
  // Articulations in order of first appearance (sim.js:99-104).
  std::vector<std::pair<int64_t, std::vector<uint32_t>>> art_joints;
  std::map<int64_t, size_t> art_index;
  for (uint32_t j = 0; j < NJ; j++) {
    const int64_t a = jart[j].i();
    auto it = art_index.find(a);
    if (it == art_index.end()) {
      art_index[a] = art_joints.size();
      art_joints.push_back({a, {}});
      it = art_index.find(a);
    }
    art_joints[it->second].second.push_back(j);
  }
  std::vector<int> body_kind(NB, 1), body_art(NB, -1), body_link(NB, -1);
  std::vector<Art> arts;
  std::vector<Link> links;
  std::vector<Dof> dofs;
  // Solver flags of the scene, then the caller's (sim.js:105-107).
  auto so_flag = [&](const char* k) { return flag(o_solver, k) || (!(o_solver && o_solver->get(k)) && flag(Ssolver, k)); };
  const bool limits_on = so_flag("enable_joint_limits");
  std::vector<double> q0, tq0, tqd0;
  std::vector<uint32_t> loops;
  const JV* pdmp = opt(&J, "passive_damping");
  const JV* spk = opt(&J, "spring_stiffness");
  const JV* spr = opt(&J, "spring_ref");
  const JV* flc = opt(&J, "friction_load_coefficient");
  const JV* tqd = opt(&J, "target_qd");
  const JV* tq_src = flag(&J, "target_q") ? J.get("target_q") : &jq;
  const JV* dd = opt(&J, "dof_dim");
  const bool jfric = so_flag("enable_joint_friction"), jvlim = so_flag("enable_joint_velocity_limits");
  for (auto& aj : art_joints) {
    const std::vector<uint32_t>& js = aj.second;
    if (aj.first < 0) { loops.insert(loops.end(), js.begin(), js.end()); continue; }
    if (js.size() == 1 && (jtype[js[0]].i() == JT_FREE || jtype[js[0]].i() == JT_DISTANCE)) continue;
    const uint32_t a = (uint32_t)arts.size();
    const uint32_t link_start = (uint32_t)links.size(), dof_start = (uint32_t)dofs.size();
    std::map<int64_t, int> local_link;
    for (uint32_t j : js) {
      int t = (int)jtype[j].i();
      if (t == JT_DISTANCE) t = JT_FREE;
      const uint32_t b = (uint32_t)jchild[j].i();
      const int l = (int)links.size();
      local_link[b] = l;
      int parent_link = -1;
      if (jparent[j].i() >= 0) {
        auto it = local_link.find(jparent[j].i());
        parent_link = it == local_link.end() ? -1 : it->second;
      }
      if (!(t == JT_FIXED || t == JT_REVOLUTE || t == JT_PRISMATIC || t == JT_BALL || t == JT_FREE || t == JT_D6))
        fail("joint type " + std::to_string(t) + " is not supported yet");
      const uint32_t ndof = (uint32_t)(qd_start[j + 1].i() - qd_start[j].i());
      const uint32_t nq = (uint32_t)(q_start[j + 1].i() - q_start[j].i());
      const uint32_t dof = (uint32_t)dofs.size(), qs = (uint32_t)q0.size();
      const bool scalar = t == JT_REVOLUTE || t == JT_PRISMATIC || t == JT_D6;
      for (uint32_t k = 0; k < ndof; k++) {
        const size_t qd = (size_t)qd_start[j].i() + k;
        Dof D{};
        const double lo = need(J, "lower")[qd].num(), hi = need(J, "upper")[qd].num();
        D.limited = (limits_on && scalar && lo > -1e5 && hi < 1e5) ? 1 : 0;
        D.armature = is_kin(b) ? 1e9 : need(J, "armature")[qd].num();
        D.ke = need(J, "ke")[qd].num();
        D.kd = need(J, "kd")[qd].num();
        D.effort = need(J, "effort")[qd].num();
        D.lower = lo;
        D.upper = hi;
        D.link = (uint32_t)links.size();
        D.damping = (pdmp && pdmp->truthy()) ? elem_or(pdmp, qd, 0.0) : 0.0;
        D.friction = jfric ? need(J, "friction")[qd].num() : 0.0;
        const JV& ax = need(J, "axis")[qd];
        for (int c = 0; c < 3; c++) D.axis[c] = ax[c].num();
        D.scalar = scalar;
        D.springKe = (scalar && spk && spk->truthy()) ? elem_or(spk, qd, 0.0) : 0.0;
        D.springRef = (spr && spr->truthy()) ? elem_or(spr, qd, 0.0) : 0.0;
        D.loadCoef = (jfric && scalar) ? ((flc && flc->truthy()) ? elem_or(flc, qd, 0.0) : 0.0) : 0.0;
        const double vl = need(J, "vel_limit")[qd].num();
        D.velLimit = (scalar && jvlim && vl < 1e5) ? vl : -1.0;
        dofs.push_back(D);
        tqd0.push_back(tqd ? (*tqd)[qd].num() : 0.0);
      }
      for (uint32_t k = 0; k < nq; k++) {
        P.q_map[q_start[j].i() + k] = (uint32_t)q0.size();
        q0.push_back(jq[(size_t)q_start[j].i() + k].num());
      }
      for (uint32_t k = 0; k < ndof; k++) P.dof_map[qd_start[j].i() + k] = dof + k;
      for (uint32_t k = 0; k < ndof; k++) tq0.push_back(scalar ? (*tq_src)[(size_t)q_start[j].i() + k].num() : 0.0);
      const bool parent_movable = parent_link >= 0 && links[parent_link].movable;
      uint32_t nlin = 0;
      if (dd && dd->truthy() && j < dd->size() && (*dd)[j].truthy()) nlin = (uint32_t)(*dd)[j][0].num();
      links.push_back(Link{t, parent_link, dof, ndof, nlin, qs, b, j, ndof > 0 || parent_movable});
      body_kind[b] = 2;
      body_art[b] = (int)a;
      body_link[b] = l;
    }
    arts.push_back(Art{link_start, (uint32_t)links.size() - link_start, dof_start, (uint32_t)dofs.size() - dof_start});
  }
  const uint32_t NA = (uint32_t)arts.size(), NL = (uint32_t)links.size(), ND = (uint32_t)dofs.size();
  // Mimics (sim.js:160-172).
  std::vector<Mimic> mimics;
  auto add_mimic = [&](int64_t f, int64_t r, double c0, double c1) {
    const int64_t n = qd_start[(size_t)f + 1].i() - qd_start[(size_t)f].i();
    for (int64_t k = 0; k < n; k++) {
      auto fd = P.dof_map.find(qd_start[(size_t)f].i() + k), ld = P.dof_map.find(qd_start[(size_t)r].i() + k);
      const int a_ = body_art[(size_t)jchild[(size_t)f].i()];
      if (fd == P.dof_map.end() || ld == P.dof_map.end() || a_ != body_art[(size_t)jchild[(size_t)r].i()])
        fail("mimic joints must share an articulation");
      const uint32_t d0 = arts[(size_t)a_].dofStart;
      mimics.push_back(Mimic{(uint32_t)a_, fd->second - d0, ld->second - d0, c0, c1,
                             P.q_map.at(q_start[(size_t)f].i() + k), P.q_map.at(q_start[(size_t)r].i() + k)});
    }
  };
  if (const JV* mj = opt(&J, "mimic_joint"))
    for (size_t f = 0; f < mj->size(); f++)
      if ((*mj)[f].num() >= 0)
        add_mimic((int64_t)f, (*mj)[f].i(), need(J, "mimic_coeffs")[f][0].num(), need(J, "mimic_coeffs")[f][1].num());
  if (const JV* ms = opt(&S, "mimics"))
    for (const JV& m : ms->a)
      if (flag(&m, "enabled"))
        add_mimic(need(m, "follower").i(), need(m, "leader").i(), need(m, "c0").num(), need(m, "c1").num());

  // Hulls and their unique edges (sim.js:180-209).
  const JV& all_shapes = need(S, "shapes");
  std::vector<const JV*> shapes;
  for (const JV& s : all_shapes.a)
    if (flag(&s, "hull") || flag(&s, "plane")) shapes.push_back(&s);
  std::map<int64_t, uint32_t> hull_index;
  std::vector<const JV*> hulls;
  for (const JV* s : shapes) {
    if (!flag(s, "hull")) continue;
    const JV& h = need(*s, "hull");
    const int64_t key = need(need(h, "verts"), "off").i();
    if (!hull_index.count(key)) {
      hull_index[key] = (uint32_t)hulls.size();
      hulls.push_back(&h);
    }
  }
  const uint32_t NS = (uint32_t)shapes.size(), NH = (uint32_t)hulls.size();
  uint64_t n_verts = 0, n_faces = 0, n_fv = 0;
  for (const JV* h : hulls) {
    n_verts += (uint64_t)need(*h, "nv").i();
    n_faces += (uint64_t)need(*h, "nf").i();
    n_fv += (uint64_t)need(need(*h, "face_verts"), "n").i();
  }
  struct Edge { uint32_t a, b, f0, f1; };
  std::vector<std::vector<Edge>> hull_edges;
  for (const JV* h : hulls) {
    const std::vector<uint32_t> fs = bin.view<uint32_t>(need(*h, "face_start"));
    const std::vector<uint32_t> fv = bin.view<uint32_t>(need(*h, "face_verts"));
    const uint32_t nf = (uint32_t)need(*h, "nf").i();
    if (fs.size() < (size_t)nf + 1) fail("hull face_start too short");
    std::map<uint64_t, std::vector<uint32_t>> faces;
    std::vector<std::pair<std::pair<uint32_t, uint32_t>, uint64_t>> edges;
    for (uint32_t f = 0; f < nf; f++) {
      const uint32_t n = fs[f + 1] - fs[f];
      for (uint32_t i = 0; i < n; i++) {
        const uint32_t a_ = fv.at(fs[f] + i), b_ = fv.at(fs[f] + (i + 1) % n);
        const uint64_t key = (uint64_t)std::min(a_, b_) * 65536u + std::max(a_, b_);
        faces[key].push_back(f);
        if (a_ < b_) edges.push_back({{a_, b_}, key});
      }
    }
    std::vector<Edge> out;
    for (auto& e : edges) out.push_back(Edge{e.first.first, e.first.second, faces[e.second].front(), faces[e.second].back()});
    hull_edges.push_back(std::move(out));
  }
  uint64_t n_edges = 0;
  for (auto& e : hull_edges) n_edges += e.size();
  const double target_frames = num_or(&S, "target_frames", 0.0), driven = num_or(&S, "driven", 0.0);
  const uint64_t path_floats = (uint64_t)(target_frames * driven);

  // statF / statU layouts (sim.js:212-237).
  std::vector<std::pair<std::string, double>> C;
  std::map<std::string, uint64_t> SF, SU;
  uint64_t off = 0;
  const std::pair<const char*, uint64_t> sf_parts[] = {
      {"SF_BODY", (uint64_t)NB * 8}, {"SF_SHAPE", (uint64_t)NS * 7}, {"SF_HAABB", (uint64_t)NH * 2},
      {"SF_VERTS", n_verts}, {"SF_FPLANE", n_faces}, {"SF_LINK", (uint64_t)std::max(NL, 1u) * 6},
      {"SF_DOF", (uint64_t)std::max(ND, 1u) * 5}, {"SF_PATH", (path_floats + 3) / 4},
      {"SF_LOOP", (uint64_t)std::max<size_t>(loops.size(), 1) * 5}, {"SF_MIMIC", (uint64_t)std::max<size_t>(mimics.size(), 1) * 2},
      {"SF_CTRL", 1}};
  for (auto& kv : sf_parts) { SF[kv.first] = off; off += kv.second; }
  std::vector<float>& sf = P.statF;
  sf.assign(off * 4, 0.0f);
  uint64_t uoff = 0;
  const std::pair<const char*, uint64_t> su_parts[] = {
      {"SU_HULL", (uint64_t)NH * 4}, {"SU_FACE", n_faces * 2}, {"SU_FV", n_fv}, {"SU_HEDGE", (uint64_t)NH * 2},
      {"SU_EDGE", n_edges * 4}, {"SU_ART", (uint64_t)std::max(NA, 1u) * 4}, {"SU_ACON", (uint64_t)std::max(NA, 1u)},
      {"SU_FILTER", ((uint64_t)NS * NS + 31) / 32}};
  for (auto& kv : su_parts) { SU[kv.first] = uoff; uoff += kv.second; }
  std::vector<uint32_t>& su = P.statU;
  su.assign(uoff, 0u);

  // Collision filter bitset (sim.js:235-255): explicit filter pairs, then shapes whose worlds or
  // groups do not meet.
  {
    std::map<size_t, uint32_t> index;
    for (size_t i = 0; i < all_shapes.size(); i++)
      if (flag(&all_shapes[i], "hull") || flag(&all_shapes[i], "plane")) {
        const uint32_t k = (uint32_t)index.size();
        index[i] = k;
      }
    const uint64_t base = SU["SU_FILTER"];
    auto set = [&](uint64_t a_, uint64_t b_) {
      const uint64_t bit = a_ * NS + b_;
      su[base + (bit >> 5)] |= 1u << (bit & 31u);
    };
    if (const JV* fl = opt(&S, "filters"))
      for (const JV& pr : fl->a) {
        auto ia = index.find((size_t)pr[0].i()), ib = index.find((size_t)pr[1].i());
        if (ia == index.end() || ib == index.end()) continue;
        set(ia->second, ib->second);
        set(ib->second, ia->second);
      }
    // The rule depends on a shape's (world, group) alone and is symmetric, so it is decided once per
    // pair of distinct (world, group) classes, and bits are set only for the members of classes
    // that do not meet: O(NS + classes^2 + filtered pairs) instead of a test of every shape pair
    // (the same bits; scenes with one class set none).
    std::map<std::pair<int64_t, int64_t>, std::vector<uint32_t>> classes;  // members in ascending order
    for (uint32_t i = 0; i < NS; i++)
      classes[{(int64_t)num_or(shapes[i], "world", -1.0), (int64_t)num_or(shapes[i], "group", -1.0)}].push_back(i);
    auto meet = [](int64_t wa, int64_t ga, int64_t wb, int64_t gb) {
      const bool gm = ga != 0 && gb != 0 && (ga > 0 ? (ga == gb || gb < 0) : ga != gb);
      return (wa < 0 || wb < 0 || wa == wb) && gm;
    };
    for (auto ca = classes.begin(); ca != classes.end(); ++ca)
      for (auto cb = ca; cb != classes.end(); ++cb) {
        if (meet(ca->first.first, ca->first.second, cb->first.first, cb->first.second)) continue;
        for (uint32_t i : ca->second)
          for (uint32_t j : cb->second)
            if (i != j) { set(i, j); set(j, i); }
      }
  }

  // Bodies (sim.js:257-305).
  P.body_pose.assign((size_t)NB * 8, 0.0f);
  const JV& mass = need(bodies, "mass");
  const JV& coms = need(bodies, "com");
  const JV& inertia = need(bodies, "inertia");
  const JV& bq_all = need(bodies, "q");
  P.body_com.assign((size_t)NB * 3, 0.0);
  for (uint32_t b = 0; b < NB; b++) {
    const size_t o_ = (SF["SF_BODY"] + (size_t)b * 8) * 4;
    const double m = mass[b].num();
    const int link = body_link[b];
    const int kind = (body_kind[b] == 2 && !links[(size_t)link].movable) ? 3 : body_kind[b];
    body_kind[b] = kind;
    const bool kinematic = is_kin(b);
    sf[o_] = (float)((m > 0 && !kinematic) ? 1 / m : 0.0);
    sf[o_ + 1] = (float)kind;
    sf[o_ + 2] = (float)body_art[b];
    sf[o_ + 3] = (float)link;
    double com[3];
    for (int c = 0; c < 3; c++) { com[c] = coms[b][c].num(); P.body_com[(size_t)b * 3 + c] = com[c]; }
    sf[o_ + 4] = (float)com[0]; sf[o_ + 5] = (float)com[1]; sf[o_ + 6] = (float)com[2];
    sf[o_ + 7] = (float)std::max(m, 0.0);
    double I[9], Ii[9];
    for (int k = 0; k < 9; k++) I[k] = inertia[b][k].num();
    inv3(I, Ii);
    for (int r = 0; r < 3; r++) {
      for (int c = 0; c < 3; c++) {
        sf[o_ + 8 + r * 4 + c] = (float)I[r * 3 + c];
        sf[o_ + 20 + r * 4 + c] = kinematic ? 0.0f : (float)Ii[r * 3 + c];
      }
      sf[o_ + 8 + r * 4 + 3] = 0.0f;
      sf[o_ + 20 + r * 4 + 3] = 0.0f;
    }
    const JV& bq = bq_all[b];
    const double q[4] = {bq[3].num(), bq[4].num(), bq[5].num(), bq[6].num()};
    double c[3];
    quat_rotate(q, com, c);
    float* bp = &P.body_pose[(size_t)b * 8];
    bp[0] = (float)(bq[0].num() + c[0]); bp[1] = (float)(bq[1].num() + c[1]); bp[2] = (float)(bq[2].num() + c[2]);
    bp[3] = 0.0f;
    for (int k = 0; k < 4; k++) bp[4 + k] = (float)q[k];
  }
  std::vector<float> radius(NB, 0.0f);
  for (const JV* s : shapes) {
    const int64_t body = need(*s, "body").i();
    if (body < 0 || flag(s, "plane")) continue;
    const double com[3] = {coms[(size_t)body][0].num(), coms[(size_t)body][1].num(), coms[(size_t)body][2].num()};
    const JV* prim = opt(s, "prim");
    const double pk = num_or(prim, "kind", 0.0);
    double sr = pk == 1 ? need(*prim, "r").num() : (pk == 2 ? need(*prim, "r").num() + need(*prim, "h").num() : 0.0);
    if (flag(s, "hull") && pk == 0) {
      const JV& h = need(*s, "hull");
      const std::vector<float> v = bin.view<float>(need(h, "verts"));
      const int64_t nv = need(h, "nv").i();
      for (int64_t i = 0; i < nv; i++) sr = std::max(sr, hypot3(v.at(i * 3), v.at(i * 3 + 1), v.at(i * 3 + 2)));
    }
    const JV& xf = need(*s, "xf");
    const double d = hypot3(xf[0].num() - com[0], xf[1].num() - com[1], xf[2].num() - com[2]);
    radius[(size_t)body] = std::max(radius[(size_t)body], (float)(d + sr));
  }
  const JV* no_grav = opt(&bodies, "no_gravity");
  const JV* ad = opt(&bodies, "angular_damping");
  for (uint32_t b = 0; b < NB; b++) {
    const size_t o_ = (SF["SF_BODY"] + (size_t)b * 8) * 4;
    sf[o_ + 11] = radius[b];
    sf[o_ + 31] = (float)((is_kin(b) ? 1 : 0) | ((no_grav && b < no_grav->size() && (*no_grav)[b].truthy()) ? 2 : 0));
    auto lim = [&](const char* k) { return elem_or(opt(&bodies, k), b, -1.0); };
    sf[o_ + 15] = (float)elem_or(ad, b, 0.05);
    sf[o_ + 19] = (float)lim("max_linear_velocity");
    sf[o_ + 23] = (float)lim("max_angular_velocity");
    sf[o_ + 27] = (float)lim("max_depenetration_velocity");
  }

  // Reduction groups (sim.js:306-313): shapes of one body with equal material share a group.
  std::vector<uint32_t> rgroup;
  {
    std::map<std::vector<double>, uint32_t> rkeys;
    const char* mat[] = {"mu", "restitution", "mu_torsional", "mu_rolling", "ke", "kd", "condim", "torsion_radius"};
    for (uint32_t i = 0; i < NS; i++) {
      const JV* s = shapes[i];
      std::vector<double> k;
      const int64_t body = need(*s, "body").i();
      if (body < 0) {
        k = {0.0, (double)i};
      } else {
        k = {1.0, (double)body};
        for (const char* f : mat) {
          const JV* v = opt(s, f);
          k.push_back(v ? 1.0 : 0.0);
          k.push_back(v ? v->num() : 0.0);
        }
      }
      auto it = rkeys.find(k);
      if (it == rkeys.end()) it = rkeys.emplace(k, (uint32_t)rkeys.size()).first;
      rgroup.push_back(it->second);
    }
  }
  const JV& GTn = need(S, "geo_type_names");
  const double GT_PLANE = need(GTn, "PLANE").num(), GT_SPHERE = need(GTn, "SPHERE").num(),
               GT_CAPSULE = need(GTn, "CAPSULE").num(), GT_BOX = need(GTn, "BOX").num(),
               GT_CYLINDER = need(GTn, "CYLINDER").num();
  for (uint32_t i = 0; i < NS; i++) {
    const JV* s = shapes[i];
    const size_t o_ = (SF["SF_SHAPE"] + (size_t)i * 7) * 4;
    const JV* prim = opt(s, "prim");
    const double type = need(*s, "type").num();
    const bool plane = flag(s, "plane");
    sf[o_] = (float)need(*s, "body").num();
    sf[o_ + 1] = flag(s, "hull") ? (float)hull_index.at(need(need(need(*s, "hull"), "verts"), "off").i()) : 0.0f;
    sf[o_ + 2] = (float)need(*s, "mu").num();
    sf[o_ + 3] = (float)num_or(s, "gap", 0.001);
    const JV& xf = need(*s, "xf");
    const double xfv[8] = {xf[0].num(), xf[1].num(), xf[2].num(), 0.0, xf[3].num(), xf[4].num(), xf[5].num(), xf[6].num()};
    for (int k = 0; k < 8; k++) sf[o_ + 4 + k] = (float)xfv[k];
    sf[o_ + 20] = (float)num_or_falsy(s, "ke", 0.0);
    sf[o_ + 21] = (float)num_or_falsy(s, "kd", 0.0);
    sf[o_ + 22] = (float)rgroup[i];
    sf[o_ + 23] = 0.0f;
    sf[o_ + 12] = plane ? 4.0f : (float)num_or(prim, "kind", 0.0);
    sf[o_ + 13] = (float)num_or(prim, "r", 0.0);
    sf[o_ + 14] = (float)num_or(prim, "h", 0.0);
    sf[o_ + 15] = (float)num_or_falsy(s, "torsion_radius", 0.0);
    sf[o_ + 16] = (float)num_or_falsy(s, "restitution", 0.0);
    sf[o_ + 17] = (float)num_or_falsy(s, "mu_torsional", 0.0);
    sf[o_ + 18] = (float)num_or_falsy(s, "mu_rolling", 0.0);
    sf[o_ + 19] = (float)num_or(s, "condim", 3.0);
    // geo scale: radius and half-height of spheres and capsules, half extents of boxes, radius and
    // half-height of cylinders from their hull vertices, else ones.
    double gs[3] = {1, 1, 1};
    if (type == GT_SPHERE || type == GT_CAPSULE) {
      gs[0] = need(*prim, "r").num(); gs[1] = need(*prim, "h").num(); gs[2] = 0;
    } else if (type == GT_BOX || type == GT_CYLINDER) {
      const std::vector<float> v = bin.view<float>(need(need(*s, "hull"), "verts"));
      double m[3] = {0, 0, 0};
      for (size_t k = 0; k < v.size(); k++) m[k % 3] = std::max(m[k % 3], (double)std::fabs(v[k]));
      if (type == GT_BOX) { gs[0] = m[0]; gs[1] = m[1]; gs[2] = m[2]; }
      else { gs[0] = m[0]; gs[1] = m[2]; gs[2] = 0; }
    }
    sf[o_ + 24] = (float)(plane ? GT_PLANE : type);
    for (int k = 0; k < 3; k++) sf[o_ + 25 + k] = (float)gs[k];
  }

  // Hull geometry (sim.js:334-355).
  {
    uint64_t v_off = 0, f_off = 0, fv_off = 0, e_off = 0;
    for (uint32_t hi = 0; hi < NH; hi++) {
      const JV& h = *hulls[hi];
      su[SU["SU_HEDGE"] + hi * 2] = (uint32_t)e_off;
      su[SU["SU_HEDGE"] + hi * 2 + 1] = (uint32_t)hull_edges[hi].size();
      for (size_t k = 0; k < hull_edges[hi].size(); k++) {
        const Edge& e = hull_edges[hi][k];
        uint32_t* w = &su[SU["SU_EDGE"] + (e_off + k) * 4];
        w[0] = e.a; w[1] = e.b; w[2] = e.f0; w[3] = e.f1;
      }
      e_off += hull_edges[hi].size();
      const std::vector<float> v = bin.view<float>(need(h, "verts"));
      const std::vector<float> planes = bin.view<float>(need(h, "face_planes"));
      const std::vector<uint32_t> fs = bin.view<uint32_t>(need(h, "face_start"));
      const std::vector<uint32_t> fv = bin.view<uint32_t>(need(h, "face_verts"));
      const uint32_t nv = (uint32_t)need(h, "nv").i(), nf = (uint32_t)need(h, "nf").i();
      if (v.size() < (size_t)nv * 3 || planes.size() < (size_t)nf * 4) fail("hull arrays too short");
      double lo[3] = {INFINITY, INFINITY, INFINITY}, hiB[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (uint32_t i = 0; i < nv; i++)
        for (int c = 0; c < 3; c++) {
          lo[c] = std::min(lo[c], (double)v[i * 3 + c]);
          hiB[c] = std::max(hiB[c], (double)v[i * 3 + c]);
        }
      const size_t base = (SF["SF_VERTS"] + v_off) * 4;
      for (uint32_t i = 0; i < nv; i++)
        for (int c = 0; c < 3; c++) sf[base + i * 4 + c] = v[i * 3 + c];
      const size_t hb = (SF["SF_HAABB"] + (size_t)hi * 2) * 4;
      for (int c = 0; c < 3; c++) {
        sf[hb + c] = (float)((lo[c] + hiB[c]) / 2);
        sf[hb + 4 + c] = (float)((hiB[c] - lo[c]) / 2);
      }
      uint32_t* hw = &su[SU["SU_HULL"] + hi * 4];
      hw[0] = (uint32_t)v_off; hw[1] = nv; hw[2] = (uint32_t)f_off; hw[3] = nf;
      for (uint32_t f = 0; f < nf; f++) {
        for (int c = 0; c < 4; c++) sf[(SF["SF_FPLANE"] + f_off + f) * 4 + c] = planes[f * 4 + c];
        su[SU["SU_FACE"] + (f_off + f) * 2] = (uint32_t)fv_off + fs.at(f);
        su[SU["SU_FACE"] + (f_off + f) * 2 + 1] = fs.at(f + 1) - fs.at(f);
      }
      for (size_t k = 0; k < fv.size(); k++) su[SU["SU_FV"] + fv_off + k] = fv[k];
      v_off += nv;
      f_off += nf;
      fv_off += fv.size();
    }
  }

  // Articulations (sim.js:356-393).
  const JV& Xp = need(J, "X_p");
  const JV& Xc = need(J, "X_c");
  const JV& axes = need(J, "axis");
  for (uint32_t i = 0; i < NL; i++) {
    const Link& l = links[i];
    const size_t o_ = (SF["SF_LINK"] + (size_t)i * 6) * 4;
    const JV& xp = Xp[l.joint];
    const JV& xc = Xc[l.joint];
    double ax[3] = {0, 0, 1};
    if (l.ndof == 1)
      for (int c = 0; c < 3; c++) ax[c] = axes[(size_t)qd_start[l.joint].i()][c].num();
    const double w[24] = {(double)l.type, (double)l.parent, (double)l.dof, (double)l.body, xp[0].num(), xp[1].num(),
                          xp[2].num(), (double)l.ndof, xp[3].num(), xp[4].num(), xp[5].num(), xp[6].num(),
                          xc[0].num(), xc[1].num(), xc[2].num(), (double)l.qs, xc[3].num(), xc[4].num(),
                          xc[5].num(), xc[6].num(), ax[0], ax[1], ax[2], l.type == JT_D6 ? (double)l.nlin : 0.0};
    for (int k = 0; k < 24; k++) sf[o_ + k] = (float)w[k];
  }
  for (uint32_t i = 0; i < ND; i++) {
    const Dof& d = dofs[i];
    const size_t o_ = (SF["SF_DOF"] + (size_t)i * 5) * 4;
    const double w[20] = {d.armature, d.ke, d.kd, d.effort, d.lower, d.upper, (double)d.limited, (double)d.link,
                          d.damping, d.friction, d.velLimit, d.scalar ? 1.0 : 0.0, d.axis[0], d.axis[1], d.axis[2],
                          d.loadCoef, d.springKe, d.springRef, 0, 0};
    for (int k = 0; k < 20; k++) sf[o_ + k] = (float)w[k];
  }
  for (uint32_t i = 0; i < NA; i++) {
    uint32_t* w = &su[SU["SU_ART"] + i * 4];
    w[0] = arts[i].linkStart; w[1] = arts[i].linkCount; w[2] = arts[i].dofStart; w[3] = arts[i].dofCount;
  }
  for (const Mimic& m : mimics) su[SU["SU_ACON"] + m.art] = 1u;
  for (uint32_t j : loops) su[SU["SU_ACON"] + (size_t)body_art[(size_t)jchild[j].i()]] = 1u;
  if (const JV* tg = opt(&S, "targets"))
    if (num_or(tg, "n", 0.0) != 0.0) {
      const std::vector<float> tv = bin.view<float>(*tg);
      if (SF["SF_PATH"] * 4 + tv.size() > sf.size()) fail("targets do not fit target_frames * driven");
      std::copy(tv.begin(), tv.end(), sf.begin() + (ptrdiff_t)(SF["SF_PATH"] * 4));
    }
  for (size_t i = 0; i < loops.size(); i++) {
    const uint32_t j = loops[i];
    const int64_t t = jtype[j].i();
    if (t != JT_BALL && t != JT_REVOLUTE) fail("loop joint type " + std::to_string(t) + " is not supported yet");
    const bool world = jparent[j].i() < 0;
    const int pl = world ? -1 : body_link[(size_t)jparent[j].i()];
    const int cl = body_link[(size_t)jchild[j].i()];
    if (cl < 0 || (!world && (pl < 0 || body_art[(size_t)jparent[j].i()] != body_art[(size_t)jchild[j].i()])))
      fail("loop joints must close inside one articulation or to the world");
    const JV& xp = Xp[j];
    const JV& xc = Xc[j];
    double ax[3] = {0, 0, 1};
    if ((size_t)qd_start[j].i() < axes.size())
      for (int c = 0; c < 3; c++) ax[c] = axes[(size_t)qd_start[j].i()][c].num();
    const double qp[4] = {xp[3].num(), xp[4].num(), xp[5].num(), xp[6].num()};
    const double qc[4] = {xc[3].num(), xc[4].num(), xc[5].num(), xc[6].num()};
    double ap[3], ac[3];
    quat_rotate(qp, ax, ap);
    quat_rotate(qc, ax, ac);
    const size_t o_ = (SF["SF_LOOP"] + i * 5) * 4;
    const double w[20] = {(double)pl, (double)cl, (double)body_art[(size_t)jchild[j].i()], t == JT_REVOLUTE ? 1.0 : 0.0,
                          xp[0].num(), xp[1].num(), xp[2].num(), 0, xc[0].num(), xc[1].num(), xc[2].num(), 0,
                          ap[0], ap[1], ap[2], 0, ac[0], ac[1], ac[2], 0};
    for (int k = 0; k < 20; k++) sf[o_ + k] = (float)w[k];
  }
  for (size_t i = 0; i < mimics.size(); i++) {
    const Mimic& m = mimics[i];
    const size_t o_ = (SF["SF_MIMIC"] + i * 2) * 4;
    const double w[8] = {(double)m.art, (double)m.f, (double)m.l, m.c1, (double)m.fq, (double)m.lq, m.c0, 0};
    for (int k = 0; k < 8; k++) sf[o_ + k] = (float)w[k];
  }
  uint32_t ctrl_kind = 0, ctrl_a = 0, ctrl_b = 0;
  if (const JV* ctrl = opt(&S, "control"))
    if (ctrl->truthy() && str_or(ctrl, "type", "") == "fader") {
      ctrl_kind = 1;
      ctrl_a = P.q_map.at(need(*ctrl, "fader_q").i());
      ctrl_b = P.dof_map.at(need(*ctrl, "wheel_v").i());
      sf[SF["SF_CTRL"] * 4] = (float)need(*ctrl, "travel").num();
      sf[SF["SF_CTRL"] * 4 + 1] = (float)need(*ctrl, "max_speed").num();
    }

  // Capacities and solver flags (sim.js:395-477).
  std::map<std::string, double> cp = {{"MAXP", 16384}, {"MAXC", 8192}, {"MAXU", 2048}, {"UH", 4096},
                                      {"WH", 16384}, {"MAXDENSE", 512}, {"AH", 4096}};
  if (const JV* caps = opt(o_in, "capacities"))
    for (auto& kv : caps->o)
      if (cp.count(kv.first)) cp[kv.first] = kv.second.num();
  const uint32_t MAXP = (uint32_t)cp["MAXP"], MAXC = (uint32_t)cp["MAXC"], MAXU = (uint32_t)cp["MAXU"],
                 UH = (uint32_t)cp["UH"], WH = (uint32_t)cp["WH"], MAXDENSE = (uint32_t)cp["MAXDENSE"],
                 AH = (uint32_t)cp["AH"];
  const uint32_t ncolw = (uint32_t)num_or(o_in, "colorWords", 2.0);
  // Solver values: defaults, then the scene's, then the caller's.
  auto sv = [&](const char* k) -> const JV* {
    if (o_solver) { const JV* v = o_solver->get(k); if (v) return v; }
    if (Ssolver) { const JV* v = Ssolver->get(k); if (v) return v; }
    return nullptr;
  };
  auto svn = [&](const char* k, double def) { const JV* v = sv(k); return v ? v->num() : def; };  // present key wins
  auto svnn = [&](const char* k, double def) { const JV* v = sv(k); return (v && !v->is_null()) ? v->num() : def; };
  auto svf = [&](const char* k) { const JV* v = sv(k); return v && v->truthy(); };
  auto svs = [&](const char* k) { const JV* v = sv(k); return (v && v->kind == JV::Str) ? v->s : std::string(); };
  auto svnull = [&](const char* k) { const JV* v = sv(k); return !v || v->is_null(); };
  double warm_start = opt(o_in, "warmStart") ? opt(o_in, "warmStart")->num() : (svf("contact_warmstart") ? 1.0 : 0.0);
  const double iters = o_iterations;
  const double fpi = svn("contact_friction_position_iterations", -1);
  const char* FMODES[] = {"fixed_normal", "bisection", "bisection_desaxce", "coulomb_newton"};
  const std::string fm = svs("friction_mode").empty() ? "fixed_normal" : svs("friction_mode");
  int fmode = -1;
  for (int k = 0; k < 4; k++)
    if (fm == FMODES[k]) fmode = k;
  if (fmode < 0) fail("friction_mode " + fm + " is not supported");
  const std::string pco = svs("propagation_color_order");
  if (!(pco.empty() || pco == "contact" || pco == "longest_first"))
    fail("propagation_color_order " + pco + " is not supported");
  if (!svnull("enable_bilateral_preelimination") && svf("enable_bilateral_preelimination"))
    fail("enable_bilateral_preelimination=true is not supported");
  if (!svnull("propagation_same_articulation_rows") && svf("propagation_same_articulation_rows"))
    fail("propagation_same_articulation_rows=true is not supported");
  if (!svnull("update_mass_matrix_interval") && svn("update_mass_matrix_interval", 1) != 1)
    fail("update_mass_matrix_interval other than 1 is not supported");
  const JV* fab = sv("friction_anchor_beta");
  const bool ang_art = svf("enable_torsional_rolling_friction");
  if (ang_art && fab && !fab->is_null() && fab->num() > 0)
    fail("enable_torsional_rolling_friction needs friction_anchor_beta=0");
  const bool compliance = svf("contact_compliance");
  const double anchor_beta = (fmode > 0 || ang_art || compliance) ? 0.0 : ((fab && !fab->is_null()) ? fab->num() : 0.2);
  const double fr_mut = svnn("free_rigid_torsional_friction", -1), fr_mur = svnn("free_rigid_rolling_friction", -1);
  bool cond4 = false, tors_on = false;
  for (const JV& s : all_shapes.a) {
    if (num_or(&s, "condim", 3.0) >= 4) cond4 = true;
    if (num_or_falsy(&s, "torsion_radius", 0.0) > 0) tors_on = true;
  }
  const bool ang_on = ang_art || fr_mut > 0 || fr_mur > 0 || cond4;
  const bool fshared = svf("contact_friction_shared_anchor");
  const bool nest = svf("nesterov_momentum");
  const uint32_t PO = ang_on ? 34 : 19;
  const uint32_t FMO = PO + ((anchor_beta > 0 || fshared) ? 4 : 0);
  const uint32_t TO = FMO + (fmode > 0 ? 2 : 0);
  const uint32_t EO = TO + (tors_on ? 5 : 0);
  const uint32_t CO = EO + (ang_art ? 4 : 0);
  const uint32_t MO = CO + (compliance ? 1 : 0);
  const uint32_t ROWS = MO + (nest ? 2 : 0);
  std::vector<std::pair<std::string, double>> Pl = {{"P_BODY", 0}, {"P_SHAPE", NB * 2.0},
                                                    {"P_AABB", NB * 2.0 + NS * 2.0}, {"P_PREV", NB * 2.0 + NS * 4.0}};
  std::vector<std::pair<std::string, double>> Sd;
  uint64_t so = 0;
  const std::pair<const char*, uint64_t> sched_parts[] = {
      {"S_HKEY", UH}, {"S_HCNT", UH}, {"S_SLOT2U", UH}, {"S_CSLOT", MAXC}, {"S_CLOCAL", MAXC}, {"S_USIZE_TMP", MAXU},
      {"S_UKEY", MAXU}, {"S_USIZE", MAXU}, {"S_USTART", (uint64_t)MAXU + 1}, {"S_CSTART", (uint64_t)ncolw * 32 + 2},
      {"S_META", 8}, {"S_CORDER", MAXC}, {"S_RK0", MAXC}, {"S_RK1", MAXC}, {"S_RK2", MAXC}, {"S_KEPT", MAXC},
      {"S_OSTART", MAXU}, {"S_LEAD", MAXC}, {"S_SLOT", (uint64_t)MAXC * 26}, {"S_ROWOF", MAXC}, {"S_RUNIT", MAXC},
      {"S_PCOL", MAXC}, {"S_PORD", MAXC}, {"S_UTC", MAXU}, {"S_UTP", MAXU}, {"S_UF", (uint64_t)NB + NA},
      {"S_UFF", (uint64_t)NB + NA}, {"S_RCON", MAXC}, {"S_WWIN", WH}, {"S_UWOFF", UH}, {"S_WALK", MAXC},
      {"S_WSLOT", (uint64_t)MAXC + MAXDENSE}};
  for (auto& kv : sched_parts) { Sd.push_back({kv.first, (double)so}); so += kv.second; }
  const uint32_t NQ = (uint32_t)q0.size();
  uint32_t NDA = 1;
  for (const Art& a_ : arts) NDA = std::max(NDA, a_.dofCount);
  const uint32_t DHDR = 25, DPS = DHDR + 6 * NDA;
  std::vector<std::pair<std::string, double>> Al;
  std::map<std::string, uint64_t> A;
  uint64_t ao = 0;
  const std::pair<const char*, uint64_t> art_parts[] = {
      {"A_Q", NQ}, {"A_QD", ND}, {"A_QDH", ND}, {"A_INT", ND}, {"A_TGT", ND}, {"A_TGTV", ND}, {"A_LIM", 2ull * ND},
      {"A_DRV", ND}, {"A_JFL", ND}, {"A_JF", ND}, {"A_BF", (uint64_t)NB * 8}, {"A_SLP", ((uint64_t)NB + NA) * 4},
      {"A_FRIC", ND}, {"A_HINV", ND}, {"A_LINK", (uint64_t)std::max(NL, 1u) * LB}, {"A_SNAP", (uint64_t)NB * 8 + ND},
      {"A_VLG", ND + (uint64_t)NB * 6}, {"A_AVL", NA}, {"A_LG", ND}, {"A_RL", ND}, {"A_RLN", NA},
      {"A_ULOAD", anchor_beta > 0 ? MAXU : 0}, {"A_DENSE", (uint64_t)MAXDENSE * DPS}};
  for (auto& kv : art_parts) { A[kv.first] = ao; Al.push_back({kv.first, (double)ao}); ao += std::max<uint64_t>(kv.second, 1); }
  std::vector<uint32_t> depth;
  uint32_t maxpath = 1, maxlp = 1, jm = 3;
  for (const Link& l : links) {
    depth.push_back(l.parent >= 0 ? depth[(size_t)l.parent] + 1 : 1);
    maxpath = std::max(maxpath, depth.back());
    if (l.ndof > 3) jm = 6;
  }
  for (const Art& a_ : arts) maxlp = std::max(maxlp, a_.linkCount);
  bool jfl = false;
  for (const Dof& d : dofs) jfl = jfl || d.loadCoef > 0;
  const double jl_gap = svnull("joint_limit_activation_gap") ? 0.05 : svn("joint_limit_activation_gap", 0.05);
  const JV* lin_v = opt(&bodies, "max_linear_velocity");
  const JV* ang_v = opt(&bodies, "max_angular_velocity");
  auto combine = [&](const char* k) {
    const char* names[] = {"average", "min", "multiply", "max"};
    const JV* v = o_solver && o_solver->get(k) ? o_solver->get(k) : (Ssolver ? Ssolver->get(k) : nullptr);
    const std::string s = (v && v->truthy() && v->kind == JV::Str) ? v->s : "average";
    for (int i = 0; i < 4; i++)
      if (s == names[i]) return (double)i;
    fail(std::string(k) + " " + s + " is not supported");
  };
  C = {{"TGT_HELD", flag(&S, "targets_held") ? 1 : 0}, {"NEST", nest ? 1 : 0}, {"MO", (double)MO}, {"NB", (double)NB},
       {"NBP", (double)std::max(NB, 1u)}, {"NBP2", std::max(NB, 1u) * 2.0}, {"NCOLW", (double)ncolw},
       {"NCOL", ncolw * 32.0}, {"NS", (double)NS}, {"NA", (double)NA}, {"NAP", (double)std::max(NA, 1u)},
       {"NL", (double)NL}, {"ND", (double)ND}, {"NDP", (double)std::max(ND, 1u)}, {"NLOOP", (double)loops.size()},
       {"NMIMIC", (double)mimics.size()}, {"CTRL_KIND", (double)ctrl_kind}, {"CTRL_A", (double)ctrl_a},
       {"CTRL_B", (double)ctrl_b}, {"NLP", (double)std::max(NL, 1u)}, {"NDA", (double)NDA}, {"JDIM", 3.0 * NDA},
       {"MAXDENSE", (double)MAXDENSE}, {"DHDR", (double)DHDR}, {"DPS", (double)DPS}, {"MAXP", (double)MAXP},
       {"MAXC", (double)MAXC}, {"MAXU", (double)MAXU}, {"UH", (double)UH}, {"WH", (double)WH}, {"ROWS", (double)ROWS},
       {"PO", (double)PO}, {"FMO", (double)FMO}, {"FMODE", (double)fmode}, {"PATCH", anchor_beta > 0 ? 1.0 : 0.0},
       {"F_ANCHOR_BETA", anchor_beta}, {"EXTRA", (anchor_beta > 0 || fshared) ? 1.0 : 0.0},
       {"SHARED", svf("contact_shared_anchor") ? 1.0 : 0.0}, {"FSHARED", fshared ? 1.0 : 0.0},
       {"F_CFM", svn("cfm", 1e-6)}, {"F_OMEGA", svn("relaxation", 1)}, {"F_SPEC", svn("contact_speculative_scale", 1)},
       {"F_GAP_GATE", svnn("contact_gap_gate", 1e30)}, {"F_FGAP", svnn("contact_friction_gap_max", 1e30)},
       {"F_FSCALE", svn("contact_friction_scale", 1)}, {"F_REST_SPEED", svn("restitution_velocity_threshold", 0.5)},
       {"REST", ((sv("enable_restitution") ? svf("enable_restitution") : true) && !compliance) ? 1.0 : 0.0},
       {"PWG", 1024}, {"CSB", 1024}, {"CTI", svs("row_schedule") == "contact_then_internal" ? 1.0 : 0.0},
       {"SLEEP", svf("enable_sleeping") ? 1.0 : 0.0}, {"F_SLEEP_LIN", svnn("sleep_linear_threshold", 0.05)},
       {"F_SLEEP_ANG", svnn("sleep_angular_threshold", 0.15)}, {"F_SLEEP_TIME", svnn("sleep_quiet_time", 0.5)},
       {"DRIVE_ROWS", svs("drive_mode") == "rows" ? 1.0 : 0.0},
       {"VEL_DRIVE_ACTIVE", svs("velocity_drive_mode") == "active" ? 1.0 : 0.0},
       {"FUSE_VLIM", (sv("fuse_joint_velocity_limits") && sv("fuse_joint_velocity_limits")->kind == JV::Bool &&
                      !sv("fuse_joint_velocity_limits")->b) ? 0.0 : 1.0},
       {"VLIM_ON", jvlim ? 1.0 : 0.0}, {"ART_F64", so_flag("articulation_fp64") ? 1.0 : 0.0},
       {"FSTART", fpi < 0 ? 0.0 : iters - std::min(fpi, iters)}, {"VELITERS", svn("velocity_iterations", 0)},
       {"AH", (double)AH}, {"ANG", ang_on ? 1.0 : 0.0}, {"ANG_ART", ang_art ? 1.0 : 0.0}, {"F_FR_MUT", fr_mut},
       {"F_FR_MUR", fr_mur}, {"JFL", jfl ? 1.0 : 0.0}, {"TORS", tors_on ? 1.0 : 0.0}, {"TO", (double)TO},
       {"EO", (double)EO}, {"PYRAMID", svs("torsional_rolling_friction_cone") == "pyramidal" ? 1.0 : 0.0},
       {"CO", (double)CO}, {"COMPL", compliance ? 1.0 : 0.0},
       {"F_CREEP", sv("torsional_rolling_friction_creep_speed") && sv("torsional_rolling_friction_creep_speed")->truthy()
                       ? sv("torsional_rolling_friction_creep_speed")->num() : 0.0},
       {"F_BP_CELL", svn("body_pair_cell_size", 0.06)}, {"LONGEST_FIRST", pco == "longest_first" ? 1.0 : 0.0},
       {"SG", 1}, {"SG32", 1}, {"F_VLIM_FRAC", svn("velocity_limit_activation_fraction", 0)},
       {"F_JL_GAP", std::min(jl_gap, 1e30)}, {"F_JL_SPEED", svnull("joint_limit_activation_gap") ? 2.0 : 0.0},
       {"VLIM_FREE", ((lin_v && lin_v->truthy()) || (ang_v && ang_v->truthy())) ? 1.0 : 0.0},
       {"JT_REVOLUTE", JT_REVOLUTE}, {"JT_PRISMATIC", JT_PRISMATIC}, {"JT_BALL", JT_BALL}, {"JT_FREE", JT_FREE},
       {"JT_D6", JT_D6}, {"FRICTION_COMBINE", combine("friction_combine")},
       {"RESTITUTION_COMBINE", combine("restitution_combine")}, {"JM", (double)jm}, {"MAXPATH", (double)maxpath},
       {"MAXLP", (double)maxlp}};
  for (auto& kv : SF) C.push_back({kv.first, (double)kv.second});
  for (auto& kv : SU) C.push_back({kv.first, (double)kv.second});
  for (auto& kv : Pl) C.push_back(kv);
  for (auto& kv : Sd) C.push_back(kv);
  for (auto& kv : Al) C.push_back(kv);
  C.push_back({"LEN_STATF4", (double)off});
  C.push_back({"LEN_STATU", (double)uoff});
  C.push_back({"LEN_SCHED", (double)so});
  C.push_back({"LEN_ART", (double)ao});

  // Initial articulation state and body velocities (sim.js:478-502).
  P.art.assign(ao, 0.0f);
  for (uint32_t k = 0; k < NQ; k++) P.art[A["A_Q"] + k] = (float)q0[k];
  for (size_t k = 0; k < tq0.size(); k++) P.art[A["A_TGT"] + k] = (float)tq0[k];
  for (size_t k = 0; k < tqd0.size(); k++) P.art[A["A_TGTV"] + k] = (float)tqd0[k];
  P.body_vel.assign((size_t)NB * 8, 0.0f);
  const JV* tw = opt(&bodies, "twist");
  if (tw)
    for (size_t b = 0; b < tw->size() && b < NB; b++) {
      const JV& t = (*tw)[b];
      if (t.is_null() || body_kind[b] != 1) continue;
      float* v = &P.body_vel[b * 8];
      v[0] = (float)t[0].num(); v[1] = (float)t[1].num(); v[2] = (float)t[2].num(); v[3] = 0;
      v[4] = (float)t[3].num(); v[5] = (float)t[4].num(); v[6] = (float)t[5].num(); v[7] = 0;
    }
  for (const Link& l : links) {
    const JV* t = (tw && l.body < tw->size()) ? &(*tw)[l.body] : nullptr;
    if (l.type != JT_FREE || l.parent >= 0 || !t || !t->truthy()) continue;
    const JV& bq = bq_all[l.body];
    const double q[4] = {bq[3].num(), bq[4].num(), bq[5].num(), bq[6].num()};
    const double com[3] = {coms[l.body][0].num(), coms[l.body][1].num(), coms[l.body][2].num()};
    double rc[3];
    quat_rotate(q, com, rc);
    const double w[3] = {(*t)[3].num(), (*t)[4].num(), (*t)[5].num()};
    const double v[3] = {(*t)[0].num() - (w[1] * rc[2] - w[2] * rc[1]), (*t)[1].num() - (w[2] * rc[0] - w[0] * rc[2]),
                         (*t)[2].num() - (w[0] * rc[1] - w[1] * rc[0])};
    float* dst = &P.art[A["A_QD"] + l.dof];
    for (int k = 0; k < 3; k++) { dst[k] = (float)v[k]; dst[3 + k] = (float)w[k]; }
  }
  // writeParams inputs (sim.js:625-639).
  const JV& grav = need(S, "gravity");
  const double fps = need(S, "fps").num();
  C.push_back({"PARAM_fps", fps});
  C.push_back({"PARAM_substeps", o_substeps});
  C.push_back({"PARAM_iterations", o_iterations});
  C.push_back({"PARAM_baumgarte", svn("baumgarte", 0.2)});
  for (int k = 0; k < 3; k++) C.push_back({"PARAM_gravity" + std::to_string(k), grav[k].num()});
  C.push_back({"PARAM_warm", warm_start * svn("contact_warmstart_decay", 1)});
  C.push_back({"PARAM_target_frames", target_frames});
  C.push_back({"PARAM_driven", driven});
  C.push_back({"PARAM_integral_count", num_or(&S, "integral_count", 0.0)});
  C.push_back({"PARAM_reg", compliance ? 0.0 : o_reg});

  P.C = C;
  P.constants.clear();
  for (auto& kv : C) P.constants += kv.first + "=" + fmt_num(kv.second) + "\n";
  P.NB = NB; P.NS = NS; P.NA = NA; P.NL = NL; P.ND = ND; P.NQ = NQ;
  P.link_body.clear();
  for (const Link& l : links) P.link_body.push_back(l.body);
  P.joint_q.clear();
  for (const JV& v : jq.a) P.joint_q.push_back((float)v.num());
  P.joint_qd_count = NJ ? (uint32_t)qd_start[NJ].i() : 0u;
  P.free_joints.clear();
  for (uint32_t j = 0; j < NJ; j++) {
    const int64_t t = jtype[j].i();
    if ((t != JT_FREE && t != JT_DISTANCE) || P.q_map.count(q_start[j].i())) continue;
    P.free_joints.push_back({(uint32_t)jchild[j].i(), (uint32_t)q_start[j].i(), (uint32_t)qd_start[j].i()});
  }
}

}  // namespace

bool pack(const JV& scene, const uint8_t* bin, size_t bin_len, const JV* opts, Packed& out, std::string& err) {
  try {
    if (scene.kind != JV::Obj) fail("scene.json is not an object");
    pack_impl(scene, Bin{bin, bin_len}, (opts && opts->kind == JV::Obj) ? opts : nullptr, out);
  } catch (const Fail& f) {
    err = f.msg;
    return false;
  } catch (const std::exception& e) {
    err = std::string("malformed scene: ") + e.what();
    return false;
  }
  return true;
}

}  // namespace scene
}  // namespace steel
