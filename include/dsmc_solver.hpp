// C++ host interface over the dsmc_b200 C ABI, mirroring the reference's
// solver API: dsmc::DSMCSolver (include/dsmc_base.h:40-80) with
// Init / SetModel / InitSystemState / RunSimulationStep / DoBenchmark /
// DumpStatistics / SampleStatistics, settings_t::readFromFile/readFromCmdLine
// (include/sim_settings.h:32-69) and CreateSolver (kernels/dsmc_base.cu:221-233).
// Failures throw std::runtime_error, as the reference's checkCUDAErrorAndThrow
// does (kernels/dsmc_kernel.cu:2066-2072).
#ifndef DSMC_SOLVER_HPP
#define DSMC_SOLVER_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "dsmc_b200.h"

namespace dsmc_b200 {

inline void check(int status, const dsmc_handle* h, const char* what) {
  if (status != DSMC_OK) {
    std::string m = std::string(what) + ": " + dsmc_status_string(status);
    const char* e = dsmc_last_error(h);
    if (e && *e) m += std::string(" (") + e + ")";
    throw std::runtime_error(m);
  }
}

// settings_t: the reference's settings plus the extensions of dsmc_config.
struct settings_t {
  dsmc_config cfg;
  float maxRunTime = -1.0f;
  settings_t() { dsmc_config_default(&cfg); }
  void readFromFile(const char* filename) { check(dsmc_config_read_xml(filename, &cfg), nullptr, "readFromFile"); }
  void readFromCmdLine(int argc, char** argv) {
    check(dsmc_config_from_args(argc, (const char* const*)argv, &cfg, &maxRunTime), nullptr,
          "readFromCmdLine");
  }
  uint32_t getCellsCount() const {
    return (uint32_t)cfg.grid_dim[0] * cfg.grid_dim[1] * cfg.grid_dim[2];
  }
};

// Per-cell sampled statistics (statistics_t, include/statistics.h:31-37) in FP64.
struct statistics_t {
  double numInSample;
  double xyzSum[3];
  double velMag;
};

// A triangle mesh with the grid resolution used to bin it (Model + the dims
// passed to Model::CreateGrid).
struct Model {
  std::vector<float> vertices;   // 3 per vertex
  std::vector<uint32_t> indices; // 3 per triangle
  std::vector<float> faceNormals;  // 3 per triangle, optional
  int gridDim[3] = {5, 5, 20};

  bool LoadRaw(const char* fname) {
    uint32_t nv = 0, nt = 0;
    if (dsmc_read_raw_mesh(fname, nullptr, &nv, nullptr, &nt, nullptr) != DSMC_OK) return false;
    vertices.resize(3 * (size_t)nv);
    indices.resize(3 * (size_t)nt);
    faceNormals.resize(3 * (size_t)nt);
    return dsmc_read_raw_mesh(fname, vertices.data(), &nv, indices.data(), &nt, faceNormals.data()) == DSMC_OK;
  }
  void CreateGrid(int x, int y, int z) { gridDim[0] = x; gridDim[1] = y; gridDim[2] = z; }
  void MoveModel(float dx, float dy, float dz) {
    for (size_t i = 0; i < vertices.size(); i += 3) {
      vertices[i] += dx; vertices[i + 1] += dy; vertices[i + 2] += dz;
    }
  }
};

class DSMCSolver {
 public:
  DSMCSolver() = default;
  ~DSMCSolver() { if (h_) dsmc_destroy(h_); }
  DSMCSolver(const DSMCSolver&) = delete;
  DSMCSolver& operator=(const DSMCSolver&) = delete;

  void Init(const settings_t& s) {
    if (h_) { dsmc_destroy(h_); h_ = nullptr; }
    settings_ = s;
    check(dsmc_create(&s.cfg, &h_), nullptr, "Init");
  }
  void SetModel(const Model& m) {
    check(dsmc_set_mesh(h_, m.vertices.data(), (uint32_t)(m.vertices.size() / 3), m.indices.data(),
                        (uint32_t)(m.indices.size() / 3),
                        m.faceNormals.empty() ? nullptr : m.faceNormals.data(), m.gridDim),
          h_, "SetModel");
  }
  uint32_t InitSystemState(const float streamVel[3]) {
    uint32_t n = 0;
    check(dsmc_init_state(h_, streamVel, &n), h_, "InitSystemState");
    return n;
  }
  // The reference's -mt start (include/gpu_dsmc.inl:341-368): twister records
  // of `path` with SEED's chain, InitMaximums, then InitMersenneTwisters; the
  // collisions draw from the cells' twisters from then on.
  void UseTwisters(const char* path, uint32_t seed = 999) {
    std::vector<uint32_t> cfg(4 * (size_t)settings_.getCellsCount());
    check(dsmc_read_twisters(path, seed, settings_.getCellsCount(), cfg.data()), nullptr,
          "UseTwisters (twister file)");
    check(dsmc_set_twisters(h_, cfg.data(), nullptr, 1), h_, "UseTwisters");
  }
  void RunSimulationStep(float dt) { check(dsmc_step(h_, dt, 1), h_, "RunSimulationStep"); }
  void DoBenchmark(uint32_t itn, float dt) {
    check(dsmc_step_graph(h_, dt, (int)itn), h_, "DoBenchmark");
    check(dsmc_sync(h_), h_, "DoBenchmark");
  }
  void DumpStatistics(const char* path) { check(dsmc_dump_statistics(h_, path), h_, "DumpStatistics"); }
  // Per-cell statistics and the collision totals (selections, collisions, sum g).
  std::vector<statistics_t> SampleStatistics(double collStat[3]) {
    check(dsmc_get_totals(h_, collStat), h_, "SampleStatistics");
    std::vector<double> s(5 * (size_t)settings_.getCellsCount());
    check(dsmc_read_cell_sums(h_, s.data(), nullptr), h_, "SampleStatistics");
    std::vector<statistics_t> out(settings_.getCellsCount());
    for (size_t c = 0; c < out.size(); c++) {
      out[c].numInSample = s[5 * c];
      out[c].xyzSum[0] = s[5 * c + 1];
      out[c].xyzSum[1] = s[5 * c + 2];
      out[c].xyzSum[2] = s[5 * c + 3];
      out[c].velMag = s[5 * c + 4];
    }
    return out;
  }
  dsmc_info Info() {
    dsmc_info i;
    check(dsmc_get_info(h_, &i), h_, "Info");
    return i;
  }
  dsmc_handle* handle() { return h_; }

 private:
  dsmc_handle* h_ = nullptr;
  settings_t settings_;
};

enum SolverType { SolverGPU, SolverGPUVBO, SolverCPU };

// CreateSolver: only the GPU solver exists (the reference returns 0 for the
// CPU solver and its VBO variant needs OpenGL).
inline DSMCSolver* CreateSolver(SolverType t) {
  return t == SolverGPU ? new DSMCSolver() : nullptr;
}

}  // namespace dsmc_b200

#endif
