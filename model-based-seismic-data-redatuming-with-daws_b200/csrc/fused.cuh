// Fused time-step kernels (stencil_fused.cu): two kernels per time step for a
// batch of shots sharing one model.
//   fused_p_step: pressure stencil + Hicks injection (gather form) + stage-B
//                 extended source + p = px + pz + free surface, and the
//                 deferred store of the previous step's velocity history;
//   fused_v_step: velocity stencil + stage-B extended sources + free surface,
//                 the deferred store of this step's pressure history, and the
//                 receiver / datum Hicks gathers in extra CTAs.
// Histories are FP32 or FP16 with one power-of-two scale per shot, step and
// field, chosen from that step's max |value| (reduced by the kernel that
// produces the field and applied by the kernel that reads it next).
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "kernels.cuh"

namespace daw {

enum FusedMode { FM_FWD = 0, FM_STAGE_A = 1, FM_STAGE_B = 2, FM_STAGE_B_ES = 3 };

constexpr int kAmaxSlots = 32;  // spread of the max-|x| atomics
// Bits of the device error flag (FusedLaunch::err).
constexpr unsigned kErrTimeout = 1u;    // a bounded tile-copy wait ran out
constexpr unsigned kErrNonFinite = 2u;  // NaN or Inf in a stage-A history field

struct ShotDevice {
  float *px, *pz, *vx, *vz, *p;  // extended-grid state [n2e][ld]
  // The one-kernel-per-step path (stencil_step.cu) alternates between two
  // state sets: {px, pz, vx, vz} above and {px2, pz2, vx2, vz2}.
  float *px2, *pz2, *vx2, *vz2;
  void* hist;                    // [nt][3][n2][n1h] (float or __half)
  unsigned* amax;                // [nt][3][kAmaxSlots] max-|x| bit patterns
  const float* amp;              // wavelet (forward) or res(nt,nr) (stage A)
  int amp_stride;                // 0 for the wavelet, nt for res
  InjMapDev inj;                 // source (forward) or receiver (stage A) map
  StationsDev rec;               // receivers for the gathers
  float* out;                    // sis(nt,nr) (forward / stage B)
  int out_reverse;               // 1: row nt-it (MINRES operator output)
  StationsDev datum;             // datum receivers (may be empty)
  float* red;                    // datum gather (nt, ndatum), accumulated (+=)
  float* wf;                     // optional (n1,n2,nt) pressure history
  int wf_acc;                    // 1: wf += p (final esource), 0: wf = p
  int nt;                        // this shot's record length
  int type_src, type_rec;
  int active;                    // 0 = skip this shot
  double* cost;                  // optional sum of 0.5*sp^2 (final esource)
};

// 2-D tensor maps of one shot's fields for the TMA kernels (box sizes in
// stencil_tma.cu): vx/vz/px/pz/p with their stencil halos, and kappa.
struct alignas(64) TmaMaps {
  CUtensorMap vx19, vz72, px, pz, p72, vx16, vz16, kap, hist;
};

// Tensor maps of one shot for the one-kernel-per-step path (box sizes in
// stencil_step.cu, which depend on the tile width): the four state fields of
// both state sets and kappa with the halo of a fused pressure + velocity
// update, and the history boxes of stage B (pressure with its halo, the
// velocities on the tile).
struct alignas(64) StepMaps {
  CUtensorMap vx[2], vz[2], px[2], pz[2], kap, histp, histv;
};

struct FusedLaunch {
  const ShotDevice* shots;  // device array
  int nshots;
  int hist_fp16;
  int n1h;                  // history leading dimension
  int chunk;                // 0: TMA kernels; 1, 2, 4: columns per thread (register kernels)
  int max_rec, max_datum;   // largest station counts (gather CTAs)
  const TmaMaps* maps;      // device array, one per shot (TMA kernels)
  unsigned* err;            // raised by a bounded wait that ran out
  int persist_p, persist_v; // persistent grid sizes of the TMA kernels
  // Stage B: the history buffer holds record steps hist_step0+1 .. (a window
  // of a checkpointed stage A) in its slots 0, 1, ...; 0 = the whole record.
  int hist_step0;
  // Per-shot pointers passed as kernel parameters for the first kParamShots
  // shots, so that a CTA's per-shot set-up needs one round of loads: the
  // max-|x| slots, the injection amplitudes in step-major order
  // [step][station] (the wavelet, or the transposed residual in stage A), the
  // record length and the station count of the injection.
  // One-kernel-per-step path: its tensor maps, the tile queue counter (zeroed
  // at the start of each run), the first step of the run, the state set the
  // run starts from, the tile width and the gather units per shot.
  const StepMaps* smaps;
  unsigned* qctr;
  int first, par0, tile_cols, ngath;
  int step_last;  // last stencil step of the run (the extra launch after it does none)
  unsigned long long active_mask;  // bit i: shot i (< 64) takes part in the run
  int pdl;  // TMA kernels launched with programmatic dependent launch
  // Split TMA kernels: the shots with work in this launch (an uneven batch's
  // short records end early), live[0 .. nlive-1]; the grid is spread over
  // them only.
  int nlive;
  unsigned char live[64];
  static constexpr int kParamShots = 8;
  int nparam;
  const unsigned* shot_amax[kParamShots];
  const float* shot_amp[kParamShots];
  int shot_nt[kParamShots];
  int shot_nsta[kParamShots];
};

// TMA kernels (stencil_tma.cu)
int tma_tiles(const Grid& g);
// Persistent grid sizes: the pressure kernels' (one for all modes), the
// velocity kernels' minimum, and the velocity kernel's per instantiation
// (index mode * 2 + fp16).
void tma_prepare(int* persist_p, int* persist_v, int* persist_v_mode);
// One bounded mbarrier wait that nothing completes: raises kErrTimeout in
// *err after `budget` cycles.
void tma_wait_selftest(unsigned* err, long long budget, cudaStream_t st);
void tma_p_step(const Grid& g, const ModelDev& m, const FusedLaunch& L, int mode, int it,
                cudaStream_t st);
void tma_v_step(const Grid& g, const ModelDev& m, const FusedLaunch& L, int mode, int it,
                cudaStream_t st);
bool tma_encode_maps(const Grid& g, const float* vx, const float* vz, const float* px,
                     const float* pz, const float* p, const float* kap, const void* hist,
                     int hist_fp16, int n1h, int nsteps, TmaMaps* out);

// Stage-A flush at it = nt+1 is folded into fused_p_step (it may exceed a
// shot's nt by one in stage A).
void fused_p_step(const Grid& g, const ModelDev& m, const FusedLaunch& L, int mode, int it,
                  cudaStream_t st);
void fused_v_step(const Grid& g, const ModelDev& m, const FusedLaunch& L, int mode, int it,
                  cudaStream_t st);
int fused_warps(const Grid& g, int chunk);

// One kernel per time step (stencil_step.cu): the pressure update of step it,
// recomputed on the velocity stencil's halo, then the velocity update, from
// state set (par0 + it - first) & 1 into the other set; plus, for step it - 1,
// the stage-A history stores and the receiver / datum gathers.  Steps run
// first .. last + 1, the extra launch doing only the work of the last step.
// Tile widths: 16 or 32 columns.
struct StepConfig {
  int tile_cols = 32;  // 16 or 32
  int ctas_per_sm = 0; // 0 = as many as fit
};
// Dynamic shared memory and resident CTAs per SM of the instantiation
// (mode, fp16, tile width); call once per device outside graph capture.
void step_prepare();
int step_occupancy(int mode, bool fp16, int tile_cols);
int step_tiles(const Grid& g, int tile_cols);
void step_launch(const Grid& g, const ModelDev& m, const FusedLaunch& L, int mode, int it,
                 int grid, cudaStream_t st);
bool step_encode_maps(const Grid& g, float* const st[2][4], const float* kap, const void* hist,
                      int hist_fp16, int n1h, int nsteps, int tile_cols, StepMaps* out);

}  // namespace daw
