// Timing driver for the reference's legacy 2-D CPU solver, the CPU code the
// reference ships for DSMC (test and baseline infrastructure only; never
// linked by the product).
//
// It links the reference's own src/dsmc_cpu.cpp, src/mtwister.cpp and
// src/genmtrand.c, compiled unchanged from the reference tree (oracle/Makefile,
// `make ref`), and runs their step as the functions ship:
//   UpdateGridCPU    (src/dsmc_cpu.cpp:176-187)  cell lists of the 30 x 18 grid
//   ComputeNanbuCPU  (src/dsmc_cpu.cpp:194-222)  Nanbu collisions per cell
//   IntegrateCPU     (src/dsmc_cpu.cpp:131-174)  free flight and wall bounces
// after GenerateInitialSpeedsPerCellCPU (src/dsmc_cpu.cpp:241-262).  The grid
// and the constants are compile-time (include/dsmc.h:27-56); nothing in the
// reference calls these functions (CreateSolver returns 0 for SolverCPU,
// kernels/dsmc_base.cu:221-233).
//
// Parameter file.  InitTwisters (src/mtwister.cpp:38-59) reads 64-byte
// mt_struct records (include/dci.h), but the shipped data/MersenneTwister.dat
// holds 65,536 of the GPU's 16-byte records (matrix_a, mask_b, mask_c, seed;
// kernels/mtwister.cu:46-68, include/MersenneTwister.h:31).  Read as 64-byte
// records, nn and mm are parameter bits and sgenrand_mt writes far past the
// 19-word state: the process crashes.  The driver therefore writes the first
// 4096 records into the layout mtwister.cpp expects, with the generator's own
// parameters (w = 32, n = 19, m = 9, r = 1, tempering shifts 12/7/15/18;
// include/MersenneTwister.h:32-40), and hands that file to InitTwisters.
//
// Usage: dsmc_cpu_legacy <MersenneTwister.dat> <particles per cell> <seconds> <max steps> <seed>
// Prints one JSON line: particles, cells, steps, seconds, particle-timesteps/s,
// and a checksum of the final velocities.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unistd.h>
#include <vector>

#include "dsmc.h"
#include "dsmc_cpu.h"
#include "mtwister.h"

namespace {

constexpr int kTwisters = 4096;  // MT_RNG_COUNT of src/mtwister.cpp

// One record as InitTwisters reads it: the first 16 words of mt_struct.
struct CpuTwisterRecord {
  uint32_t aaa;
  int32_t mm, nn, rr, ww;
  uint32_t wmask, umask, lmask;
  int32_t shift0, shift1, shiftB, shiftC;
  uint32_t maskB, maskC;
  int32_t i;
  uint32_t pad;
};
static_assert(sizeof(CpuTwisterRecord) == 64, "InitTwisters reads 16 words per record");

bool write_cpu_records(const char* gpu_dat, const char* out_path) {
  FILE* in = std::fopen(gpu_dat, "rb");
  if (!in) return false;
  std::vector<uint32_t> words(4u * kTwisters);
  const size_t got = std::fread(words.data(), 16, kTwisters, in);
  std::fclose(in);
  if (got != static_cast<size_t>(kTwisters)) return false;
  std::vector<CpuTwisterRecord> rec(kTwisters);
  for (int k = 0; k < kTwisters; ++k) {
    CpuTwisterRecord& r = rec[k];
    std::memset(&r, 0, sizeof(r));
    r.aaa = words[4 * k + 0];
    r.maskB = words[4 * k + 1];
    r.maskC = words[4 * k + 2];
    r.mm = 9;
    r.nn = 19;
    r.rr = 1;
    r.ww = 32;
    r.wmask = 0xFFFFFFFFu;
    r.umask = 0xFFFFFFFEu;
    r.lmask = 0x1u;
    r.shift0 = 12;
    r.shift1 = 18;
    r.shiftB = 7;
    r.shiftC = 15;
  }
  FILE* out = std::fopen(out_path, "wb");
  if (!out) return false;
  const bool ok = std::fwrite(rec.data(), sizeof(CpuTwisterRecord), kTwisters, out) ==
                  static_cast<size_t>(kTwisters);
  return std::fclose(out) == 0 && ok;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 6) {
    std::fprintf(stderr, "usage: %s <MersenneTwister.dat> <particles per cell> <seconds> <max steps> <seed>\n",
                 argv[0]);
    return 2;
  }
  const unsigned ppc = static_cast<unsigned>(std::strtoul(argv[2], nullptr, 10));
  const double budget = std::strtod(argv[3], nullptr);
  const long max_steps = std::strtol(argv[4], nullptr, 10);
  const unsigned seed = static_cast<unsigned>(std::strtoul(argv[5], nullptr, 10));
  if (ppc == 0 || max_steps <= 0) {
    std::fprintf(stderr, "particles per cell and max steps must be positive\n");
    return 2;
  }
  char tmpl[] = "/tmp/dsmc_cpu_legacy_mt_XXXXXX";
  const int fd = mkstemp(tmpl);
  if (fd < 0) {
    std::perror("mkstemp");
    return 1;
  }
  close(fd);
  if (!write_cpu_records(argv[1], tmpl)) {
    std::fprintf(stderr, "cannot convert the twister parameters of %s\n", argv[1]);
    unlink(tmpl);
    return 1;
  }
  InitTwisters(tmpl, seed);
  unlink(tmpl);

  const unsigned cells = GRID_DIM_X * GRID_DIM_Y;
  const unsigned n = cells * ppc;
  std::vector<float> vel(2u * n), pos(2u * n), cols(3u * n);
  GenerateInitialSpeedsPerCellCPU(vel.data(), pos.data(), 0.f, 0.f, ppc, 0);

  auto one_step = [&]() {
    UpdateGridCPU(pos.data(), n);
    ComputeNanbuCPU(vel.data(), 0);
    IntegrateCPU(vel.data(), pos.data(), cols.data(), DSMC_DT, n);
  };
  one_step();  // warm-up: the cell lists reach their capacity
  long steps = 0;
  double seconds = 0.0;
  while (steps < max_steps && seconds < budget) {
    const auto t0 = std::chrono::steady_clock::now();
    one_step();
    seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    ++steps;
  }
  double checksum = 0.0;
  for (float v : vel) checksum += v;
  std::printf("{\"particles\": %u, \"cells\": %u, \"steps\": %ld, \"seconds\": %.6f, "
              "\"value\": %.6e, \"threads\": 1, \"checksum\": %.9e}\n",
              n, cells, steps, seconds, steps > 0 ? double(n) * steps / seconds : 0.0, checksum);
  return 0;
}
