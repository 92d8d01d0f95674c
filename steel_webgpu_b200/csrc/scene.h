// Scene files to the packed form, on the host: a JSON reader for scene.json and the packer that
// turns a loaded scene (scene.json + scene.bin, the reference's LoadedScene of sceneTypes.ts:91-99)
// into statF, statU, the constant table and the initial state (Sim.build, sim.js:95-521).
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace steel {
namespace scene {

// One JSON value.
struct JV {
  enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
  bool b = false;
  double n = 0.0;
  std::string s;
  std::vector<JV> a;
  std::vector<std::pair<std::string, JV>> o;

  const JV* get(const char* key) const;       // member or nullptr (objects only)
  bool truthy() const;                         // Python truthiness of the decoded value
  bool is_null() const { return kind == Null; }
  double num(double def = 0.0) const { return kind == Num ? n : (kind == Bool ? (b ? 1.0 : 0.0) : def); }
  int64_t i() const { return (int64_t)num(); }
  size_t size() const { return kind == Arr ? a.size() : 0; }
  const JV& operator[](size_t k) const;
};
bool parse_json(const char* text, size_t len, JV& out, std::string& err);

// A packed scene: the C ABI's steel_scene_desc contents plus the maps Sim.state() and the Newton-
// indexed setters need (sim.js:99-157, :732-763).
struct Packed {
  std::vector<std::pair<std::string, double>> C;  // constants, then PARAM_* writeParams inputs
  std::string constants;                           // "KEY=VALUE\n" text of C
  std::vector<float> statF, body_pose, body_vel, art;
  std::vector<uint32_t> statU;
  uint32_t NB = 0, NS = 0, NA = 0, NL = 0, ND = 0, NQ = 0;
  std::map<int64_t, uint32_t> dof_map, q_map;  // Newton dof / coordinate -> port dof / coordinate
  std::vector<uint32_t> link_body;             // body of each link
  std::vector<double> body_com;                // NB * 3, scene.json bodies.com
  std::vector<float> joint_q;                  // scene.json joints.q (Newton layout)
  uint32_t joint_qd_count = 0;                 // joints.qd_start[last]
  struct FreeJoint { uint32_t body, q_start, qd_start; };
  std::vector<FreeJoint> free_joints;          // free joints outside articulations (state() mirrors the body)
};
// opts: SimOptions (sim.d.ts:3-28) as JSON, may be null: substeps, iterations, regularization,
// warmStart, colorWords, solver (overrides of scene.json's solver), plus "capacities" (MAXP, MAXC,
// MAXU, UH, WH, MAXDENSE, AH) replacing the reference's fixed ones.
bool pack(const JV& scene, const uint8_t* bin, size_t bin_len, const JV* opts, Packed& out, std::string& err);

}  // namespace scene
}  // namespace steel
