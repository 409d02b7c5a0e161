// main_redatum_daw: the reference's program (src/main_redatum_DAW.f90) on the
// B200 library.  Reads redatum.par from the working directory (or argv[1]).
// Shots are block-partitioned over ranks like para_range
// (src/para_range.f90:11-22) using RANK/WORLD_SIZE from the environment, one
// process per GPU (LOCAL_RANK selects the device).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "daw_b200.h"
#include "daw_internal.h"

static int env_int(const char* k, int dflt) {
  const char* v = std::getenv(k);
  return v ? std::atoi(v) : dflt;
}

int main(int argc, char** argv) {
  const std::string dir = argc > 1 ? argv[1] : ".";
  const int rank = env_int("RANK", 0), size = env_int("WORLD_SIZE", 1);
  const int dev = env_int("LOCAL_RANK", 0);
  const auto t0 = std::chrono::steady_clock::now();
  daw_handle* h = nullptr;
  int rc = daw_create(&h, dev);
  if (rc != DAW_OK) {
    std::fprintf(stderr, "daw_create failed (%d): no usable sm_100 GPU\n", rc);
    return 2;
  }
  daw::ParFile pf;
  std::string err;
  if (!daw::read_parfile(dir + "/redatum.par", &pf, &err)) {
    std::fprintf(stderr, "%s\n", err.c_str());
    daw_destroy(h);
    return 1;
  }
  // count shots from the acquisition header
  std::vector<int32_t> st, rt;
  int nsrc = 0, nrec = 0;
  if (!daw::read_acquisition(dir + "/" + pf.name_acqui, pf.h, pf.npml, pf.ofs, &st, &nsrc, &rt,
                             &nrec, &err)) {
    std::fprintf(stderr, "%s\n", err.c_str());
    daw_destroy(h);
    return 1;
  }
  if (rank == 0) {
    std::printf(" Run mode: %d\n Number of sources and receivers %d %d\n", pf.mode, nsrc, nrec);
  }
  const int w1 = nsrc / size, w2 = nsrc % size;  // para_range
  const int ista = rank * w1 + 1 + (rank < w2 ? rank : w2);
  int iend = ista + w1 - 1;
  if (w2 > rank) iend += 1;
  if (iend >= ista) rc = daw_run_parfile(h, dir.c_str(), ista, iend);
  if (rc != DAW_OK) std::fprintf(stderr, "error %d: %s\n", rc, daw_last_error(h));
  daw_destroy(h);
  const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (rank == 0) std::printf(" ELAPSED TIME = %.3f\n", el);
  return rc == DAW_OK ? 0 : 1;
}
