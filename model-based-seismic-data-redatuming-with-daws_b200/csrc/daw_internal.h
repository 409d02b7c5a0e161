// Internal declarations shared by the host C++ and CUDA sources of
// libdaw_b200.so.  Not part of the public ABI (include/daw_b200.h).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "daw_b200.h"

namespace daw {

constexpr int kRad = 10;           // Hicks support radius (irad)
constexpr int kTap = 2 * kRad + 1; // taps per axis
constexpr int kTile = kTap * kTap; // 441 coefficients per station
constexpr int kNAlpha = 100;       // sub-grid positions per axis (nalpha)

// ---------------------------------------------------------------------------
// Host-side Hicks coefficients (hicks.cpp)
// ---------------------------------------------------------------------------
// 21x21 monopole tile of one station, tile[(i1+10) + 21*(i2+10)], with the
// free-surface anti-mirroring for nalpha_frees > 0.
void hicks_tile(int ialpha1, int ialpha2, int nfs, float* tile);
// subsourcekws for a 2-D position (z, x): out5 = ix1, ix2 (1-based, physical),
// ialpha1, ialpha2, nalpha_frees.
void hicks_locate(float z, float x, float h, int ofs, int32_t out5[5]);

// Parameter file / acquisition (hicks.cpp)
struct ParFile {
  int mode = 0;
  std::string name_true, name_init, name_acqui, name_src;
  float flow = 0, fhig = 0, llow = 0, lhig = 0;
  int n1 = 0, n2 = 0, npml = 0, nt = 0;
  float h = 0, dt = 0, dto = 0;
  int type_src = 0, type_rec = 0, ofs = 0;
  float mu = 0;
  int oio = 0;
  float error = 0, maxiter = 0;
};
bool read_parfile(const std::string& path, ParFile* pf, std::string* err);
bool read_acquisition(const std::string& path, float h, int npml, int ofs,
                      std::vector<int32_t>* src_tab, int* nsrc,
                      std::vector<int32_t>* rec_tab, int* nrec, std::string* err);
std::string shot_name(int i);  // subname: 5-digit zero padded

// ---------------------------------------------------------------------------
// Device-side descriptors
// ---------------------------------------------------------------------------
struct Grid {
  int n1, n2, npml, n1e, n2e;
  int ld;        // leading dimension of extended-grid fields (floats), %64 == 0
  int ofs;
  float h, dt, dtdx;
  __host__ __device__ size_t ext_elems() const { return (size_t)ld * n2e; }
  __host__ __device__ size_t int_elems() const { return (size_t)n1 * n2; }
  // Fused-path history layout [step][field][i2p][hist_rows]: extended row i1
  // is stored at row i1 - hist_base, hist_base = npml rounded down to a
  // multiple of 8, so a lane's (even, odd) row pair is aligned and a tile's
  // first row is a 16-byte-aligned tensor-copy coordinate.
  __host__ __device__ int hist_base() const { return npml & ~7; }
  __host__ __device__ int hist_rows() const { return ((npml - (npml & ~7)) + n1 + 7) / 8 * 8; }
};

struct ModelDev {
  float* kap = nullptr;                  // [n2e][ld] kappa = vp^2
  float* d1a = nullptr; float* d1b = nullptr;   // damp1a, damp1b (n1e)
  float* d2a = nullptr; float* d2b = nullptr;   // damp2a, damp2b (n2e)
  float* d1a1 = nullptr; float* d2a1 = nullptr; // damp1a1, damp2a1
  float* bw1 = nullptr; float* bw2 = nullptr;   // dtdx*1*damp1b1, dtdx*1*damp2b1
  // The same profiles packed for one load per row / column:
  // prow[i1] = (d1a, d1a1, d1b, bw1), pcol[i2] = (d2a, d2a1, d2b, bw2).
  float4* prow = nullptr;
  float4* pcol = nullptr;
  // With a density other than 1 (else null): the buoyancy-weighted update
  // coefficients dtdx*bu1*damp1b1 and dtdx*bu2*damp2b1 and the buoyancy
  // bu = 1/rho itself, on the extended grid ([n2e][ld]).
  float* rbw1 = nullptr;
  float* rbw2 = nullptr;
  float* rbue = nullptr;
};

// A set of Hicks stations (sources or receivers) on the device.
struct StationsDev {
  int n = 0;
  int* ix1 = nullptr;   // 1-based indices (extended grid for sources/receivers)
  int* ix2 = nullptr;
  float* tile = nullptr;  // n * 441
};

// Gather-form injection map of a station set on the extended grid: for every
// touched grid point the (station, coefficient) contributions in station
// order, so the per-point sum has the reference's accumulation order.
struct InjMapDev {
  int npts = 0, nent = 0;
  int* pt = nullptr;       // linear index i1 + ld*i2 (0-based) of each touched point
  int* ptr = nullptr;      // npts+1 entry offsets
  int* sta = nullptr;      // station of each entry
  float* coef = nullptr;   // coefficient of each entry
  // Column-band view for the fused kernels.
  int* col_lo = nullptr;   // n2e: first touched row (0-based) or INT_MAX
  int* col_hi = nullptr;   // n2e: last touched row or -1
  int* col_base = nullptr; // n2e: dense-row index of row col_lo
  int* rowptr = nullptr;   // per dense row: [begin, end) entry offsets
  float2* ent = nullptr;   // per entry: (coefficient, station index as int bits)
  int nsta = 0;            // stations of the map
};

// ---------------------------------------------------------------------------
// Simple device memory owner.
// ---------------------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

struct Options {
  int preset = 1;
  int history_fp16 = 1;
  int scalars_fp64 = 1;
  int fused = 1;
  int graph = 1;
  int skip_dead_op = 0;
  int max_batch = 0;
  int chunk = 0;
  int checkpoint = 0;  // stage-A history window in steps (0 = automatic)
  int step = 0;        // TMA kernels: 0 = p and v kernels, 1 = one kernel per step, 2 = autotuned
  int pdl = 0;         // TMA kernels: programmatic dependent launch between time steps
  int tile_cols = 0;   // one-kernel-per-step tiles: 16 or 32 columns, 0 = autotuned
  int ctas_per_sm = 0; // one-kernel-per-step CTAs per SM, 0 = autotuned
};

}  // namespace daw
