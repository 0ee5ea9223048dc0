// dsmc_bench: the reference's -benchmark run (kernels/dsmc.cu:308-470) on the
// B200 library.  Same flags (-f, -benchmark, -no-geometry, -density, -dt,
// -run-for) plus:
//   -raw FILE             load a .raw mesh (the reference hard-codes data/ares.raw)
//   -icosphere L R X Y Z  icosphere mesh, subdivision L, radius R, centre X Y Z
//   -geom-grid X Y Z      geometry grid dims (reference: 5 5 20)
//   -move X Y Z           translate the mesh (reference: 0 0 -3)
//   -steps N              run N steps instead of -run-for
//   -stats FILE           statistics output (default statistics.txt)
//   -mt                   the reference's Mersenne-Twister collisions, twister
//                         records from data/MersenneTwister.dat (the reference's path)
//   -mt-file FILE         another twister parameter file
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dsmc_solver.hpp"

int main(int argc, char** argv) {
  try {
    // -mt and -mt-file are taken here; the settings parser sees the rest
    bool mt = false;
    std::string mt_file = "data/MersenneTwister.dat";
    std::vector<char*> rest;
    for (int i = 0; i < argc; i++) {
      if (i > 0 && !strcmp(argv[i], "-mt")) {
        mt = true;
      } else if (i > 0 && !strcmp(argv[i], "-mt-file") && i + 1 < argc) {
        mt = true;
        mt_file = argv[++i];
      } else {
        rest.push_back(argv[i]);
      }
    }
    dsmc_b200::settings_t s;
    s.readFromCmdLine((int)rest.size(), rest.data());
    std::string raw, stats = "statistics.txt";
    bool ico = false;
    float ico_r = 0.1f, ico_c[3] = {0, 0, 0}, mv[3] = {0, 0, 0};
    int ico_l = 3, gdim[3] = {5, 5, 20};
    long steps = -1;
    for (int i = 1; i < argc; i++) {
      if (!strcmp(argv[i], "-raw") && i + 1 < argc) raw = argv[++i];
      else if (!strcmp(argv[i], "-icosphere") && i + 5 < argc) {
        ico = true;
        ico_l = atoi(argv[++i]);
        ico_r = (float)atof(argv[++i]);
        for (int k = 0; k < 3; k++) ico_c[k] = (float)atof(argv[++i]);
      } else if (!strcmp(argv[i], "-geom-grid") && i + 3 < argc) {
        for (int k = 0; k < 3; k++) gdim[k] = atoi(argv[++i]);
      } else if (!strcmp(argv[i], "-move") && i + 3 < argc) {
        for (int k = 0; k < 3; k++) mv[k] = (float)atof(argv[++i]);
      } else if (!strcmp(argv[i], "-steps") && i + 1 < argc) {
        steps = atol(argv[++i]);
      } else if (!strcmp(argv[i], "-stats") && i + 1 < argc) {
        stats = argv[++i];
      }
    }
    const bool geometry = !raw.empty() || ico;
    s.cfg.geometry = geometry ? 1 : 0;

    dsmc_b200::DSMCSolver solver;
    solver.Init(s);
    if (geometry) {
      dsmc_b200::Model model;
      if (!raw.empty()) {
        if (!model.LoadRaw(raw.c_str())) throw std::runtime_error("Unable to load model");
      } else {
        uint32_t nv = 0, nt = 0;
        dsmc_b200::check(dsmc_mesh_icosphere(ico_l, ico_r, ico_c, nullptr, &nv, nullptr, &nt), nullptr, "mesh");
        model.vertices.resize(3 * (size_t)nv);
        model.indices.resize(3 * (size_t)nt);
        dsmc_b200::check(dsmc_mesh_icosphere(ico_l, ico_r, ico_c, model.vertices.data(), &nv,
                                             model.indices.data(), &nt), nullptr, "mesh");
      }
      model.CreateGrid(gdim[0], gdim[1], gdim[2]);
      model.MoveModel(mv[0], mv[1], mv[2]);
      solver.SetModel(model);
    }
    dsmc_info info = solver.Info();
    std::printf("Expected number of particles per cell: %u density is %g\n", info.part_per_cell,
                (double)s.cfg.density);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a);
    uint32_t n = solver.InitSystemState(s.cfg.stream_vel);
    if (mt) solver.UseTwisters(mt_file.c_str());
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    std::printf("%u samples were generated in %g ms\n", n, ms);
    long nIter = steps >= 0 ? steps : (long)(s.maxRunTime / s.cfg.dt + 1);
    if (nIter <= 0) throw std::runtime_error("give -run-for T or -steps N");
    std::printf("Starting benchmarking. Will run %ld iterations\n", nIter);
    cudaEventRecord(a);
    solver.DoBenchmark((uint32_t)nIter, s.cfg.dt);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    std::printf("Benchmark is done in %g ms\n", ms);
    info = solver.Info();
    std::printf("particle-timesteps/s: %.4g (%u particles)\n", (double)n * nIter / (ms * 1e-3),
                info.num_particles);
    solver.DumpStatistics(stats.c_str());
  } catch (std::exception& e) {
    std::fprintf(stderr, "Exception: %s\n", e.what());
    return 1;
  }
  return 0;
}
