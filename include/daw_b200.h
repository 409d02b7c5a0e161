/*
 * daw_b200.h -- C ABI of the B200 (sm_100a) DAW redatuming library.
 *
 * The boundary sits between the reference's workflow driver
 * (src/sub_redatum_DAW.f90, modes 0/1/2/3) and its wave-propagation engine
 * and MINRES solver (src/submodeling2.f90, src/sublinearminres.f90,
 * src/minresModule.f90, src/subwavefieldresample.f90).  Every entry point is
 * callable from Fortran through ISO_C_BINDING (bind(C), value arguments for
 * scalars, arrays as plain pointers):
 *   - scalars: int32_t = default INTEGER, float = default REAL, double;
 *   - arrays: column-major exactly as the reference declares them, first
 *     index fastest (sis(nt,nr), wavefield(n1,n2,nt), vp(n1,n2));
 *   - acquisition tables: (n,5) int32 column-major with the 1-based
 *     extended-grid contents subacqui builds (src/subacqui.f90:30-58):
 *     ix1+npml, ix2+npml, ialpha1, ialpha2, nalpha_frees.
 *
 * Ownership: callers own every host array and the library keeps no pointer
 * to one after a call returns.  The library owns all device memory (model,
 * Hicks tiles, wavefield state, histories, MINRES vectors) inside a handle.
 * Calls are synchronous.  A handle is bound to one GPU and is not
 * thread-safe; use one handle per host thread (one MPI rank per GPU keeps the
 * reference's rank structure).
 *
 * Errors: every int-returning call returns DAW_OK (0) or a negative
 * daw_status; daw_last_error() gives the message.  Nothing exits or throws
 * across the ABI.  There is no CPU fallback: without a usable sm_100 GPU,
 * daw_create returns DAW_ERR_NODEV.
 */
#ifndef DAW_B200_H
#define DAW_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct daw_handle daw_handle;

enum daw_status {
  DAW_OK = 0,
  DAW_ERR_ARG = -1,     /* invalid argument or inconsistent sizes */
  DAW_ERR_OOM = -2,     /* host/device allocation failed or HBM admission refused */
  DAW_ERR_CUDA = -3,    /* CUDA runtime error */
  DAW_ERR_TIMEOUT = -4, /* a bounded device-side wait ran out */
  DAW_ERR_NAN = -5,     /* non-finite value detected in a wavefield history */
  DAW_ERR_IO = -6,      /* file or parse error (driver entry points) */
  DAW_ERR_STATE = -7,   /* call order: model or acquisition not set */
  DAW_ERR_NODEV = -8    /* no usable sm_100 CUDA device */
};

/* Execution options (daw_set_option).  The two presets are the plain FP32
 * GPU port (literal kernel-per-loop port, FP32 histories, FP32 MINRES
 * scalars) and the mixed path (fused kernels, FP16 histories with per-step
 * power-of-two scales, FP64 MINRES inner products and scalars, CUDA graphs). */
enum daw_option {
  DAW_OPT_PRESET = 0,        /* 0 = plain FP32 port, 1 = mixed (default) */
  DAW_OPT_HISTORY = 1,       /* 0 = FP32 history, 1 = FP16 scaled history */
  DAW_OPT_SCALARS = 2,       /* 0 = FP32 MINRES dots/scalars, 1 = FP64 */
  DAW_OPT_FUSED = 3,         /* 0 = one kernel per reference loop, 1 = fused */
  DAW_OPT_GRAPH = 4,         /* 1 = capture time loops in CUDA graphs */
  DAW_OPT_SKIP_DEAD_OP = 5,  /* 1 = skip MINRES's unused initial operator
                                application (minresModule.f90:132); default 0 */
  DAW_OPT_MAX_BATCH = 6,     /* upper bound on shots per batched launch (0 = auto) */
  DAW_OPT_CHUNK = 7,         /* fused kernels: 0 = TMA-pipelined persistent kernels
                                (default); 1, 2 or 4 = register kernels with that
                                many columns per thread */
  DAW_OPT_CHECKPOINT = 8     /* fused kernels: stage-A history window in time steps.
                                0 (default) = the whole record when a shot's history
                                fits in device memory, else the largest window that
                                fits; K > 0 = windows of K steps.  A shot with a
                                window runs alone: stage A saves its state before each
                                window and is re-run over each window (but the last)
                                from that state while stage B consumes the windows in
                                reverse order.  No counterpart in the reference, which
                                keeps whole histories. */,
  DAW_OPT_STEP_KERNEL = 9,   /* TMA kernel family (DAW_OPT_CHUNK = 0): 0 (default) =
                                separate pressure and velocity kernels, shots per launch
                                and CTAs per SM chosen by the autotuner; 1 = one kernel
                                per time step (pressure recomputed on the velocity
                                stencil's halo, two alternating state sets), tile width
                                and CTAs per SM autotuned; 2 = the family autotuned too
                                (the windows of a checkpointed shot use the separate
                                kernels unless 1 is set) */
  DAW_OPT_TILE_COLS = 10,    /* one-kernel-per-step tiles: 16 or 32 columns of 64
                                rows; 0 (default) = chosen by the autotuner */
  DAW_OPT_CTAS_PER_SM = 11,  /* one-kernel-per-step CTAs per SM (1..3; a value above
                                what fits is lowered to the occupancy); 0 (default) =
                                chosen by the autotuner */
  DAW_OPT_PDL = 12           /* TMA kernels: 1 = programmatic dependent launch (a time
                                step's kernel starts launching while the previous one
                                drains); 0 (default) = plain stream order */
};

/* Handle lifetime ------------------------------------------------------- */
int daw_create(daw_handle** out, int32_t device);
void daw_destroy(daw_handle* h);
const char* daw_last_error(const daw_handle* h);
int daw_set_option(daw_handle* h, int32_t key, double value);
int daw_get_option(const daw_handle* h, int32_t key, double* value);

/* Model: the background/true velocity vp(n1,n2) and grid of the reference's
 * `grid` (main_redatum_DAW.f90:10-24).  Density is identically 1 as in the
 * reference (submodeling2.f90:93).  Replaces the per-call set-up of
 * submodeling2.f90:54-113 (substagger/submodext/cspongea/cspongeb). */
int daw_set_model(daw_handle* h, const float* vp, int32_t n1, int32_t n2, int32_t npml,
                  float hgrid, float dt, int32_t ofs);

/* The same with a density rho(n1,n2) (column-major; NULL = rho 1, the same
 * as daw_set_model).  The reference allocates rho and fixes it to 1
 * (submodeling2.f90:88-93, :961); this entry point passes a real density
 * through its substagger arithmetic (:1227-1270): kappa = rho vp^2 in double,
 * buoyancy 1/rho (1e10 where rho <= 0) averaged onto the staggered velocity
 * grids, and the buoyancy weight of the velocity sources (:252, :838, :845).
 * A density other than 1 runs on the plain kernels and the split TMA
 * pressure/velocity kernels; the register kernels (DAW_OPT_CHUNK != 0) and
 * the one-kernel-per-step family (DAW_OPT_STEP_KERNEL = 1) refuse it with
 * DAW_ERR_ARG, and the autotuner (DAW_OPT_STEP_KERNEL = 2) keeps to the
 * split kernels. */
int daw_set_model_rho(daw_handle* h, const float* vp, const float* rho, int32_t n1, int32_t n2,
                      int32_t npml, float hgrid, float dt, int32_t ofs);

/* Datum receivers for the on-the-fly mode-2 resampling (rec_tab of the
 * mode-2 run, sub_redatum_DAW.f90:238; table as subacqui builds it). */
int daw_set_datum(daw_handle* h, const int32_t* datum_tab, int32_t ndatum);

/* Reference-routine mirrors (host arrays; one shot per call) ------------ */

/* submodeling (submodeling2.f90:11): forward modelling with the source s
 * (nt samples, already divided by h^2 as main_redatum_DAW.f90:111 does).
 * sis(nt,nr) out; wavefield(n1,n2,nt) out or NULL. */
int daw_submodeling(daw_handle* h, const float* s, int32_t nt, const int32_t* is5,
                    int32_t type_src, int32_t type_rec, const int32_t* ir, int32_t nr,
                    float* sis, float* wavefield);

/* submodeling_adjoint_esource_data (submodeling2.f90:880): the G G^T
 * operator; res(nt,nr) in, sis(nt,nr) out. */
int daw_esource_data(daw_handle* h, const float* res, int32_t nt, int32_t type_rec,
                     const int32_t* ir, int32_t nr, float* sis);

/* submodeling_adjoint_esource (submodeling2.f90:523): sis(nt,nr) out,
 * wavefieldp(n1,n2,nt) out or NULL, *cost = sum of 0.5*sp^2 (the printed
 * `cost`, :734-744) or NULL. */
int daw_esource(daw_handle* h, const float* res, int32_t nt, int32_t type_rec,
                const int32_t* ir, int32_t nr, float* sis, float* wavefieldp, double* cost);

/* MINRES report (minresModule.f90:10-360 outputs).  log rows are
 * (itn, x(1), norm(r)/beta1, norm(A), cond(A)) per iteration. */
typedef struct daw_minres_info {
  int32_t istop, itn, nlog, log_capacity;
  double anorm, acond, rnorm, arnorm, ynorm, shift, beta1;
  double* log; /* caller array of 5*log_capacity doubles, or NULL */
} daw_minres_info;

/* sublinearminres (sublinearminres.f90:7): solve (A + fac I) x = deltadr with
 * A = time-reverse(G G^T), fac = mu*||deltadr||/||G G^T deltadr||, x0 = 0,
 * no preconditioner (the reference passes .false., :74), itnlim = maxiter,
 * rtol.  deltadr, deltade (nt,nr). */
int daw_linear_minres(daw_handle* h, const float* deltadr, int32_t nt, int32_t type_rec,
                      const int32_t* ir, int32_t nr, float mu, int32_t maxiter, float rtol,
                      float* deltade, daw_minres_info* info);

/* subwavefieldresample (subwavefieldresample.f90:1): Hicks gather of a
 * physical-grid history wavefield(n1,n2,nt) at ir(nr,5), support clipped to
 * the physical grid; sis(nt,nr) out.  Uses the handle's n1, n2, npml. */
int daw_wavefield_resample(daw_handle* h, const float* wavefield, int32_t nt,
                           const int32_t* ir, int32_t nr, float* sis);

/* filmartin2d (minresModule.f90:486): per-trace zero-padded FP64 FFT band
 * pass.  flow/fhig/llow/lhig are in/out: fhig is clamped to Nyquist and lhig
 * zeroed in place when fhig exceeds it, as the reference does (:523-527). */
int daw_filmartin2d(daw_handle* h, const float* in, int32_t nr, int32_t nt, float dt,
                    float* flow, float* fhig, float* llow, float* lhig, float* out);

/* filmartin2d on traces already in device memory, allocating nothing.  It
 * has no counterpart in the reference.  It is for callers that cannot
 * allocate GPU memory at the moment they filter: HBM already held by a shot
 * batch (admitted up to ~92 % of the device) or by a framework's caching
 * allocator, or code that must not stall other streams with the device-wide
 * synchronisation of cudaMalloc/cudaFree.
 *   d_in, d_out: (nt,nr) column-major float32 device buffers of the current
 *   device (caller-owned); band parameters in/out as in daw_filmartin2d;
 *   stream: a cudaStream_t (NULL = legacy default stream); err: optional
 *   buffer of err_len bytes for the message of a failed call.
 * Work space is one fixed 4 MiB array that every GPU where it is set up
 * holds until exit (weights for nto <= 65536, FFT space for long traces).
 * nt above 65536 is rejected with DAW_ERR_ARG.  The set-up, once per device
 * with that device current, takes the array's device address; under CUDA's
 * default lazy module loading that is also when the array and the filter
 * kernel's code are placed on the device, which can need device memory.
 * daw_create runs it for its device; on a device without a handle, make one
 * call with nr = 0 (d_in and d_out may then be NULL) before the device fills
 * up and before any stream capture.  Calls share the array, so their GPU work
 * must not overlap: calls are serialised by a lock and return after their
 * work has finished on `stream`. */
int daw_filmartin2d_noalloc(const float* d_in, int32_t nr, int32_t nt, float dt, float* flow,
                            float* fhig, float* llow, float* lhig, float* d_out, void* stream,
                            char* err, int32_t err_len);

/* Mode-1 DAW shot pipeline (sub_redatum_DAW.f90:73-156) with the mode-2
 * resampling at the datum receivers fused on the fly (:230-240) ---------- */
typedef struct daw_shot_desc {
  int32_t shot;            /* 1-based shot number (logs only) */
  int32_t nt;              /* record length of this shot */
  const float* s;          /* wavelet (nt), already divided by h^2 */
  int32_t src_tab[5];      /* src_tab(isrc,:) */
  const int32_t* rec_tab;  /* (nrec,5) */
  int32_t nrec;
  const float* dobs;       /* observed data (nt,nrec) */
  int32_t type_src, type_rec;
  float mu;                /* penalty (grid%mu) */
  int32_t maxiter;         /* MINRES itnlim */
  float rtol;              /* MINRES rtol (grid%error) */
  float band[4];           /* flow, fhig, llow, lhig for the datum filter */
} daw_shot_desc;

typedef struct daw_shot_out {   /* every pointer may be NULL */
  float* datar;        /* (nt,nrec) reduced data d(c0) */
  float* deltadr;      /* (nt,nrec) time-reversed residuals, memory order of inv%deltadr */
  float* deltade;      /* (nt,nrec) MINRES solution */
  float* dataesc;      /* (nt,nrec) scattered data */
  float* datae;        /* (nt,nrec) datar + dataesc */
  float* redatumed_raw;/* (nt,ndatum) DAW gathered at the datum, before filtering */
  float* redatumed;    /* (nt,ndatum) after filmartin2d (dataobs_redatum) */
  float* wavefield_exd;/* (n1,n2,nt) DAW history (oio=1 output) */
  double cost;         /* esource `cost` */
  daw_minres_info minres;
} daw_shot_out;

int daw_shot(daw_handle* h, const daw_shot_desc* desc, daw_shot_out* out);

/* Batched: n shots (uneven nt, receiver spreads and sources allowed) run in
 * shared launches.  The shots are taken longest record first (so a batch
 * holds similar record lengths); each batch takes the longest run of the
 * remaining shots whose device bytes (each shot's own record length and
 * receiver count) fit ~92 % of the free HBM.  outs[i] pairs with descs[i]. */
int daw_shots(daw_handle* h, int32_t n, const daw_shot_desc* descs, daw_shot_out* outs);

/* Batched forward modelling, mode 0 (sub_redatum_DAW.f90:55-72: submodeling
 * of every shot in the true model).  No history is kept, so up to 64 shots
 * share each launch.  descs[i] supplies s, nt, src_tab, rec_tab, nrec,
 * type_src, type_rec (other fields ignored); sis[i] receives that shot's
 * (nt, nrec) receiver data.  For the wavefield output (oio = 1) call
 * daw_submodeling per shot. */
int daw_submodeling_shots(daw_handle* h, int32_t n, const daw_shot_desc* descs,
                          float* const* sis);

/* Batch planning (no counterpart in the reference; no device work): *count
 * receives how many of descs[0 .. n-1], taken in order, HBM admits as one
 * batch (the rule of daw_shots), *window (nullable) the stage-A history
 * window a lone shot would use (0 = whole record). */
int daw_admit_shots(daw_handle* h, int32_t n, const daw_shot_desc* descs, int32_t* count,
                    int32_t* window);

/* Device-resident timing support: shots whose inputs were staged once with
 * daw_stage_shots run with no host transfers; results stay on the device
 * until daw_fetch_shots. ms_out (nullable) receives the device time. */
int daw_stage_shots(daw_handle* h, int32_t n, const daw_shot_desc* descs);
int daw_run_staged(daw_handle* h, float* ms_out);
int daw_fetch_shots(daw_handle* h, daw_shot_out* outs);

/* Reference workflow (main_redatum_DAW + sub_redatum_DAW): reads
 * redatum.par and its inputs from `workdir`, runs shots [first,last] (1-based,
 * inclusive; 0,0 = all) and writes the reference's output files there. */
int daw_run_parfile(daw_handle* h, const char* workdir, int32_t first, int32_t last);

/* Timing of the last pipeline call: device milliseconds by phase. */
typedef struct daw_timing {
  double forward_ms, operator_ms, minres_vec_ms, esource_ms, filter_ms, total_ms;
  double sim_fwd_ms, sim_a_ms, sim_b_ms;  /* device time of the time loops by kind */
  double steps_fwd, steps_a, steps_b;     /* time steps launched (batch-wide) */
  double shot_steps;          /* shot time steps (sum over shots of batch steps) */
  double point_updates;       /* extended-grid point updates performed */
  double hist_bytes;          /* history bytes written + read */
  int64_t kernel_launches;    /* kernels launched by the library */
  double shot_steps_fwd, shot_steps_a, shot_steps_b;  /* shot time steps by kind */
  /* TMA kernels of the last run of each mode (forward, stage A, stage B, final
   * esource), as the autotuner chose them: family (0 = separate pressure and
   * velocity kernels, 1 = one kernel per step), tile columns, CTAs per SM
   * (separate kernels: of the pressure kernel) and CTAs per SM of the
   * velocity kernel (0 for one kernel per step); zeros = not run */
  int32_t kernel_family[4], tile_cols[4], ctas_per_sm[4], ctas_per_sm_v[4];
  int32_t shots_per_launch[4]; /* shots whose time loops share one launch */
} daw_timing;
int daw_get_timing(const daw_handle* h, daw_timing* t);
void daw_reset_timing(daw_handle* h);

/* Hicks helpers on the host (no device work): the 21x21 monopole tile of
 * (ialpha1, ialpha2, nalpha_frees) with free-surface anti-mirroring
 * (kwsinc2d, src/kwsinc.f90:212-378; tile[(i1+10) + 21*(i2+10)]) and the
 * (ix1, ix2, ialpha1, ialpha2, nalpha_frees) of a (z, x) position
 * (subsourcekws, src/kwsinc.f90:582-606). */
void daw_hicks_tile(int32_t ialpha1, int32_t ialpha2, int32_t nalpha_frees, float* tile);
void daw_hicks_locate(float z, float x, float hgrid, int32_t ofs, int32_t* out5);

/* Diagnostic (no counterpart in the reference): runs one device-side
 * bounded wait that nothing completes, with a ~0.5 ms budget, and returns
 * what the library reports when a wait runs out -- DAW_ERR_TIMEOUT when the
 * failure path works.  No GPU fault is involved; the handle stays usable. */
int daw_selftest_wait_timeout(daw_handle* h);

/* Library version string. */
const char* daw_version(void);

#ifdef __cplusplus
}
#endif
#endif /* DAW_B200_H */
