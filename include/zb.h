/*
 * zb.h -- C ABI of libzb, the B200 (sm_100a) finite-volume kernels behind the
 * zoomy-b200 host package.
 *
 * Conventions
 *   - All array arguments are DEVICE pointers unless a name ends in _host.
 *   - State arrays use the reference layout (n_state, n_cells), cell axis last,
 *     one contiguous plane per state row: Q = [b | h | q_x | q_y] for 2-D SWE.
 *     Cartesian cell (i, j) (i along x, j along y) is cell i*ny + j.
 *   - dtype: ZB_F32 or ZB_F64, for every floating array of the call.
 *   - Every call takes the CUDA stream to launch on and returns 0 on success,
 *     a negative ZB_E* code for a rejected argument or a CUDA launch error.
 *     Device-side findings (non-finite or non-positive dt, troubled cells,
 *     unconverged solves) are written to the status word of the caller's
 *     zb_ctrl block and read by the host after the stream is synchronised.
 *   - No call allocates device memory.  Scratch lives in caller-provided
 *     workspace whose size the matching *_workspace_bytes call returns.
 *
 * Reference interfaces replaced (paths inside ZoomyLab/zoomy-jax):
 *   zoomy_jax/fvm/solver2/blocks.py:36-95    dt_pass + reduce_dt
 *   zoomy_jax/fvm/solver2/blocks.py:98-124   assert_dt_admissible (status bits)
 *   zoomy_jax/fvm/solver2/blocks.py:129-287  halo_bc, reconstruct, flux_pass,
 *                                            gather_update (one fused stage)
 *   zoomy_jax/fvm/solver2/march.py:126-157   stage_loop (SSP-RK2 Shu-Osher)
 *   zoomy_jax/fvm/solver_jax.py:990-1131     _explicit_hyperbolic_step + step
 *   zoomy_jax/fvm/solver_jax.py:284-369      update_qaux (KP hinv + LSQ rows)
 */
#ifndef ZB_H
#define ZB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* zb_stream_t; /* a cudaStream_t */

enum { ZB_F32 = 0, ZB_F64 = 1 };

enum {
  ZB_OK = 0,
  ZB_E_ARG = -1,      /* invalid argument (size, enum, null pointer) */
  ZB_E_CUDA = -2,     /* CUDA launch / runtime error */
  ZB_E_UNSUPPORTED = -3,
  ZB_E_TOO_LARGE = -4,      /* grid exceeds a fixed-size buffer (noalloc step, TMEM) */
  ZB_E_NOT_CONVERGED = -5   /* an iterative solve missed its tolerance */
};

/* status bits written by the kernels into zb_ctrl.status */
enum {
  ZB_ST_DT_INVALID = 1u,   /* dt non-finite or <= 0 before t_end (fatal) */
  ZB_ST_TROUBLED = 2u,     /* a cell left h >= 0 or became non-finite */
  ZB_ST_NOT_CONVERGED = 4u /* an iterative solve missed its tolerance */
};

/* boundary-condition kinds per side (reference BC.Extrapolation / Wall /
 * Periodic; tests/cases.py:115-175) */
enum { ZB_BC_EXTRAPOLATION = 0, ZB_BC_WALL = 1, ZB_BC_PERIODIC = 2 };
enum { ZB_RECON_CONSTANT = 0, ZB_RECON_CONSERVATIVE = 1, ZB_RECON_ETA = 2 };
enum { ZB_RIEMANN_RUSANOV = 0, ZB_RIEMANN_RUSANOV_HR = 1, ZB_RIEMANN_HLL_HR = 2 };
enum { ZB_LIM_MINMOD = 0, ZB_LIM_BARTH_JESPERSEN = 1, ZB_LIM_VENKATAKRISHNAN = 2,
       ZB_LIM_NONE = 3 };

/* Device control block (caller-allocated device memory, 128 bytes, 8-byte
 * aligned).  The step kernels triple-buffer the wave-speed maximum and the
 * time by phase = step index mod 3: step n reads slot n%3, writes slot
 * (n+1)%3 and clears slot (n+2)%3, so K steps run without a host sync and
 * without a race between the clearing block and the accumulating blocks. */
typedef struct {
  double amax[3];     /* max over faces of |lambda| (phase-indexed)         */
  double t[3];        /* simulation time (phase-indexed)                    */
  double dt;          /* dt taken by the last step                          */
  double mass;        /* last zb_swe2d_mass result (sum h |cell|)           */
  uint32_t status;    /* ZB_ST_* bits, sticky until the host clears them    */
  uint32_t steps;     /* steps completed (incremented by the final stage)   */
  uint32_t troubled;  /* troubled cells seen in the last step               */
  uint32_t pad;
  double reserved[6];
} zb_ctrl;

/* Scheme and physics of the Cartesian 2-D SWE step.  Plain C struct. */
typedef struct {
  int32_t nx, ny;          /* cells along x and y                         */
  double x0, y0, dx, dy;   /* origin and spacing                          */
  int32_t order;           /* 1: Euler + constant recon, 2: SSP-RK2 + MUSCL */
  int32_t recon;           /* ZB_RECON_*                                   */
  int32_t riemann;         /* ZB_RIEMANN_*                                 */
  int32_t limiter;         /* ZB_LIM_*                                     */
  int32_t bc[4];           /* left, right, bottom, top: ZB_BC_*            */
  double g;                /* gravity                                      */
  double wet_dry_eps;      /* KP hinv desingularisation                    */
  double eps_wet;          /* eta recon dry demotion (<0: none)            */
  double manning_n;        /* Manning coefficient (0: no friction)         */
  int32_t implicit_source; /* 0: explicit RK1 Manning, 1: point-implicit   */
  int32_t dim_factor;      /* d of the CFL law (2 for 2-D)                 */
  double cfl;              /* CFL safety factor                            */
  double dt_max;           /* dt cap (+inf: none)                          */
  double t_end;            /* t_end clamp (+inf: none)                     */
  int32_t degree;          /* k of the (2k+1) CFL factor                   */
  int32_t dtype;           /* ZB_F32 / ZB_F64                              */
  /* NULL, or the planes zb_swe2d_bed_prepare wrote for the b row of every
   * state stepped with this config (device memory).  Read by the fused steps
   * of the order-2 eta / HLL-HR scheme on grids without a periodic side
   * (ignored by every other scheme, by the stage API and by the ensemble);
   * the results are the same bits either way.  The caller owns the promise
   * that b has not changed since the planes were prepared. */
  const void* bed;
} zb_swe2d_cfg;

/* Library version / build info. */
const char* zb_version(void);

/* Bytes of device workspace zb_swe2d_step needs (one stage buffer of three
 * planes plus alignment padding). */
size_t zb_swe2d_workspace_bytes(const zb_swe2d_cfg* cfg);

/* Bytes of the bed planes of cfg's scheme (0 when the scheme does not read
 * them: see zb_swe2d_cfg.bed). */
size_t zb_swe2d_bed_bytes(const zb_swe2d_cfg* cfg);

/* The bathymetry's interior least-squares gradient (x, y) and limiter value,
 * three planes of the config's dtype laid out like a state row, from the b
 * row of Q.  b is constant in time (the reference steps it with a zero
 * update), so a march prepares them once and the interior body of every step
 * reads them instead of re-evaluating b's slope each stage (the reference's reconstruction
 * evaluates the gradient and limiter of every variable, b included, on every
 * call: zoomy_jax/fvm/reconstruction_jax.py:524-533, 695-708).  ZB_E_ARG for
 * a scheme without bed planes. */
int zb_swe2d_bed_prepare(const zb_swe2d_cfg* cfg, const void* Q, void* bed,
                         size_t bed_bytes, zb_stream_t stream);

/* Initialise the control block for a march starting at time t0 from state Q:
 * clears status and all slots, sets t[phase] = t0 and amax[phase] = the
 * maximum wave speed of Q.  Also creates, once per device and host thread,
 * the library's second stream that the fused step forks its boundary-strip
 * launch onto (call it outside stream capture, on the thread that will step
 * or capture; the steps themselves capture).  Each host thread has its own
 * second stream and fork / join events, so host threads may step different
 * solvers on one device at once.
 * Replaces the first dt_pass (zoomy_jax/fvm/solver2/blocks.py:36-61). */
int zb_swe2d_init(const zb_swe2d_cfg* cfg, const void* Q, zb_ctrl* ctrl,
                  int phase, double t0, zb_stream_t stream);

/* dt of the state in Q: dt_pass + reduce_dt with t_remaining = t_end - t
 * (zoomy_jax/fvm/solver2/blocks.py:36-95).  Writes ctrl->dt. */
int zb_swe2d_dt(const zb_swe2d_cfg* cfg, const void* Q, zb_ctrl* ctrl,
                double t, zb_stream_t stream);

/* One full time step, in place on Q (the b row is read, never written):
 * dt from ctrl->amax[phase] (CFL law, dt_max, t_end clamp), the hyperbolic
 * sub-step (order 2: SSP-RK2 with the KP aux refreshed between stages; order
 * 1: Euler), Manning friction, and the wave-speed maximum of the new state
 * into ctrl->amax[(phase + 1) % 3].  phase = step index mod 3.  Replaces HyperbolicSolver.step + post_step
 * (zoomy_jax/fvm/solver_jax.py:1095-1172) and MarchSolver.hyperbolic_step
 * (zoomy_jax/fvm/solver2/march.py:161-175).  Graph-capturable: no host
 * sync, no allocation. */
int zb_swe2d_step(const zb_swe2d_cfg* cfg, void* Q, void* workspace,
                  size_t workspace_bytes, zb_ctrl* ctrl, int phase,
                  zb_stream_t stream);

/* Largest grid (nx * ny) zb_swe2d_step_noalloc accepts. */
#define ZB_NOALLOC_MAX_CELLS (1u << 20)

/* zb_swe2d_step for callers that cannot allocate device memory.  No
 * counterpart in the reference.  Such callers are plugins inside a framework
 * that owns every device byte and hands them only their operands (an XLA /
 * JAX FFI custom call declared without a scratch operand, an
 * inference-engine plugin at enqueue time).  The caller passes Q and ctrl as for
 * zb_swe2d_step; the stage-1 scratch is a file-scope device array inside
 * libzb sized for ZB_NOALLOC_MAX_CELLS cells (24 MiB, held on every GPU that
 * loads the library until the process exits).  Larger grids return
 * ZB_E_TOO_LARGE without launching.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current, so
 * make that first call before any stream capture.  Nothing is allocated and
 * no library routine that allocates is called.  Every call shares the one
 * array and it keeps the last call's contents (the step overwrites every
 * scratch cell it reads, so nothing needs clearing); calls that overlap on
 * the GPU -- concurrent streams, or several host threads on one device --
 * race on it and must be serialised by the caller.  The looked-up address is
 * kept for the life of the process: do not use the library across a
 * cudaDeviceReset. */
int zb_swe2d_step_noalloc(const zb_swe2d_cfg* cfg, void* Q, zb_ctrl* ctrl,
                          int phase, zb_stream_t stream);

/* One launch of zb_swe2d_step: part 0 is the first stage (order 2) or the
 * Euler stage (order 1), part 1 the second stage (order 2) or the copy-back
 * (order 1); part -1 is the whole step.  Calling part 0 then part 1 on the
 * same stream is exactly zb_swe2d_step; the split lets a caller bracket each
 * kernel with events. */
int zb_swe2d_step_part(const zb_swe2d_cfg* cfg, void* Q, void* workspace,
                       size_t workspace_bytes, zb_ctrl* ctrl, int phase,
                       int part, zb_stream_t stream);

/* One explicit stage with a host-given dt (dt < 0: read ctrl->dt):
 * Q_out = alpha * Q0 + (1 - alpha) * (Qk + beta * dt * (L(Qk) + S(Qk))),
 * the Shu-Osher form of solver2's stage loop (zoomy_jax/fvm/solver2/
 * blocks.py:241-287, march.py:126-157).  S is the Manning source with aux
 * hinv_src (one plane; NULL: no source in the stage).  force_o1 (C bytes or
 * NULL) demotes flagged cells to constant reconstruction, the MOOD mask of
 * zoomy_jax/fvm/reconstruction_jax.py:1246-1251.  trouble_out (C bytes or
 * NULL) receives the troubled predicate h < 0 | non-finite per cell
 * (solver2/blocks.py:290-301); any troubled cell also sets ZB_ST_TROUBLED.
 * Q_out's b row is not written.  Q_out may alias Q0 but not Qk. */
int zb_swe2d_stage(const zb_swe2d_cfg* cfg, const void* Qk, const void* Q0,
                   void* Q_out, double alpha, double beta, double dt,
                   const void* hinv_src, const uint8_t* force_o1,
                   uint8_t* trouble_out, zb_ctrl* ctrl, zb_stream_t stream);

/* Source step Q += dt * S(Q, hinv0) for Manning friction, explicit RK1 or
 * point-implicit (cfg->implicit_source), with hinv0 the aux of the step's
 * input state (one plane of C values).  Replaces get_compute_source + ode.RK1
 * (zoomy_jax/fvm/solver_jax.py:373-397, 1129; zoomy_jax/fvm/ode.py:14-18)
 * and the local implicit source of the IMEX solver
 * (zoomy_jax/fvm/solver_imex_jax.py:269-342). */
int zb_swe2d_source(const zb_swe2d_cfg* cfg, void* Q, const void* hinv0,
                    double dt, zb_stream_t stream);

/* Sum of h * |cell| in float64 (deterministic two-pass reduction) into
 * ctrl->mass.  partial must hold zb_swe2d_mass_partials(cfg) doubles. */
size_t zb_swe2d_mass_partials(const zb_swe2d_cfg* cfg);
int zb_swe2d_mass(const zb_swe2d_cfg* cfg, const void* Q, double* partial,
                  zb_ctrl* ctrl, zb_stream_t stream);

/* Post-step aux rows (zoomy_jax/fvm/solver_jax.py:284-369) into Qaux (7, C):
 * [dqx/dx, dh/dx, dqy/dy, dh/dy, db/dx, db/dy, hinv], LSQ with
 * extrapolation ghosts. */
int zb_swe2d_aux(const zb_swe2d_cfg* cfg, const void* Q, void* Qaux,
                 zb_stream_t stream);

/* Diagnostic with no counterpart in the reference: the float64 quotient
 * a[i] / b[i], square root sqrt(b[i]) and reciprocal square root
 * 1 / sqrt(b[i]) as the float64 shallow-water kernels compute them (Newton
 * refinement of the hardware approximations), into out[0..n), out[n..2n) and
 * out[2n..3n) (device pointers; b > 0), for their accuracy test against IEEE
 * arithmetic. */
int zb_newton_check_f64(const double* a, const double* b, double* out, int64_t n,
                        zb_stream_t stream);

/* ── batched ensemble of Cartesian instances ─────────────────────────────── */

/* One independent instance of the ensemble (host description).  Its state
 * is (4, nx*ny) at element offset q_offset of the batch state array and its
 * stage buffer (3, nx*ny) at element offset ws_offset of the batch
 * workspace.  Every other scheme field comes from the common config. */
typedef struct {
  int32_t nx, ny;
  double dx, dy;
  int64_t q_offset;
  int64_t ws_offset;
  double manning_n;
  double t_end;
} zb_ens_instance;

/* Launch shape of the ensemble step: what zb_ens_prepare_tuned lays into the
 * work list and zb_ens_step_part_tuned launches.  No counterpart in the
 * reference (its ensemble is a Python loop over solvers); the autotuner of
 * the host package picks it by timing candidates on the actual ensemble.
 *   tile_x          tile height of the small-grid fallback (8 or 16)
 *   ctas_per_sm     persistent strip CTAs per SM: 1..4 (float32), 1..2 (float64)
 *   n_classes       size classes of instances (1..4); an instance of side
 *                   max(nx, ny) belongs to the first class whose
 *                   class_max_side is >= that side (the last class takes
 *                   every larger one); class_max_side increases
 *   edge_rows       column-EDGE chunk height per class (4..32 rows)
 *   interior_rows   interior chunk height per class (8..1024 rows) */
typedef struct {
  int32_t tile_x;
  int32_t ctas_per_sm;
  int32_t n_classes;
  int32_t class_max_side[4];
  int32_t edge_rows[4];
  int32_t interior_rows[4];
} zb_ens_tuning;

/* Device bytes of the instance table + work list for a tile height of
 * tile_x (8 or 16) cells; 0 if the configuration is not supported (the
 * ensemble runs the order-2 eta reconstruction with HR-HLL, wall or
 * extrapolation boundaries). */
size_t zb_ens_table_bytes(const zb_swe2d_cfg* common,
                          const zb_ens_instance* inst, int n_inst, int tile_x);

/* Build the per-instance parameter blocks (spacing, least-squares weights,
 * Manning, t_end) and the work list, and copy them to the device table.  The
 * call waits for all work on the current device before it copies (a table
 * that steps in flight still read is not overwritten under them) and returns
 * once the copy has landed: call at set-up, outside stream capture.  The
 * work list holds every instance's (instance, strip, row chunk) items of the single grid's full-coverage list (interior, boundary-
 * column and boundary-row bodies), and (instance, tile) items for grids
 * narrower than four cells.  *n_items_out receives the work-list length
 * (tiles + strips). */
int zb_ens_prepare(const zb_swe2d_cfg* common, const zb_ens_instance* inst,
                   int n_inst, int tile_x, void* table, size_t table_bytes,
                   int* n_items_out);

/* zb_ens_table_bytes / zb_ens_prepare with an explicit launch shape (the
 * untuned calls use one class with 32-row column-EDGE chunks, 64-row interior
 * chunks and 4 (float32) or 2 (float64) strip CTAs per SM). */
size_t zb_ens_table_bytes_tuned(const zb_swe2d_cfg* common, const zb_ens_instance* inst,
                                int n_inst, const zb_ens_tuning* tuning);
int zb_ens_prepare_tuned(const zb_swe2d_cfg* common, const zb_ens_instance* inst,
                         int n_inst, const zb_ens_tuning* tuning, void* table,
                         size_t table_bytes, int* n_items_out);

/* Reset the n_inst control blocks ctrls[0..n_inst) and seed each instance's
 * wave-speed maximum from its state (zb_swe2d_init per instance; it also
 * creates the second stream, outside stream capture). */
int zb_ens_init(const zb_swe2d_cfg* common, const void* table, int n_inst,
                const void* Q, zb_ctrl* ctrls, int phase, double t0,
                zb_stream_t stream);

/* One SSP-RK2 step of every instance: part 0 = the first stage, 1 = the
 * second, -1 = both.  Each stage is four persistent kernels: warps walking the
 * boundary-column and then the boundary-row strip items on the library's
 * second stream beside warps walking the interior strip items on `stream`,
 * then CTAs walking the tiles of grids narrower than four cells (grid <= 0
 * picks SMs x occupancy for the latter; with no such grid they exit at
 * once).  Each instance takes its own CFL dt (zb_swe2d_step semantics per
 * instance). */
int zb_ens_step_part(const zb_swe2d_cfg* common, const void* table, int n_inst,
                     int n_items, int tile_x, int grid, void* Q, void* W,
                     zb_ctrl* ctrls, int phase, int part, zb_stream_t stream);

/* zb_ens_step_part with the launch shape the table was prepared with. */
int zb_ens_step_part_tuned(const zb_swe2d_cfg* common, const void* table, int n_inst,
                           int n_items, const zb_ens_tuning* tuning, int grid, void* Q,
                           void* W, zb_ctrl* ctrls, int phase, int part,
                           zb_stream_t stream);

/* ── Chorin pressure solve ─────────────────────────────────────────────────
 * Variable-coefficient Poisson -div(c grad p) = f on an nx x ny Cartesian grid
 * (c = clip(h, cmin, cmax), harmonic face means, Dirichlet p = 0), float64
 * flexible CG preconditioned by a float32 geometric-multigrid V-cycle.
 * Replaces the pressure solve of the reference's Chorin projection
 * (zoomy_jax/fvm/solver_chorin_vam_jax.py:673-883: unpreconditioned GMRES on
 * VAM's operator) and its corrector (:885-907). */
typedef struct {
  int32_t nx, ny;
  double dx;
  double cmin, cmax;
  int32_t nu;            /* pre- and post-smoothing red-black sweeps          */
  int32_t coarse_sweeps; /* symmetric sweep pairs on the coarsest level       */
  int32_t coarsest;      /* stop coarsening at this side                      */
} zb_poisson_cfg;

/* The learned smoother: a two-level convolutional U-Net (c1 channels at full
 * resolution, c2 at half resolution; (c1, c2) one of (8, 16), (16, 16),
 * (16, 32), (24, 48) -- the last has 52.6k parameters -- tanh) with bf16
 * weights and float32 accumulation.  Given a residual r it returns the
 * correction s dx^2 / c * U([r / s, c / cmax]) (s = RMS of r, c the cell
 * coefficient): a learned local smoother in place of the red-black
 * sweeps of the level-0 multigrid smoothing.  Counterpart of the learned
 * V-cycle smoother of the reference (zoomy_jax/gnn_blueprint/
 * vcycle_structured_gnn.py:74-122, graph_mp_multibranch.py:9-16).  Weights are
 * [Cout][Cin][3][3] per layer, layers e1 (2->c1), e2 (c1->c1), m1 (c1->c2),
 * m2 (c2->c2), o1 (c2+c1->c1), out (c1->1), concatenated. */
typedef struct zb_smoother {
  int32_t c1, c2;
  const void* w;          /* bf16 weights, device                            */
  const float* b;         /* float32 biases, device                          */
  float cmax;             /* coefficient normalisation                       */
  void* act;              /* activation workspace, device                    */
  size_t act_bytes;       /* >= zb_smoother_workspace_bytes(c1, c2, nx, ny)  */
  int32_t max_nx, max_ny;
} zb_smoother;

/* Convolution engine of the U-Net's forward and data-gradient passes:
 * 1 = tcgen05 implicit GEMM (bf16 operands, float32 accumulation; default;
 * zb_smoother_apply's activations in a chunked bf16 layout, 8 channels per
 * 16 bytes), 2 = the same GEMM staging float32 planar activations everywhere
 * (the same bits as 1), 0 = CUDA-core direct convolution (float32 operands).
 * Returns the previous setting (process-wide; any other value only queries). */
int zb_unet_conv_impl(int impl);

/* Error word of the tensor-core kernels: non-zero when a bounded wait timed
 * out (the tile's outputs were not written).  Synchronous; clear != 0 resets. */
int zb_unet_status(int clear);

/* Parameters of a (c1, c2) U-Net: returns weights + biases. */
size_t zb_unet_param_count(int c1, int c2, size_t* n_weights, size_t* n_biases);
size_t zb_smoother_workspace_bytes(int c1, int c2, int nx, int ny);

/* x_out = x_in + S(f - A x_in) on one nx x ny grid (x_in may be NULL for a
 * zero start; x_out may alias x_in); cx, cy are the float32 face
 * coefficients, r_scratch holds nx*ny floats. */
int zb_smoother_apply(const zb_smoother* smoother, const float* f,
                      const float* x_in, float* x_out, const float* cx,
                      const float* cy, float* r_scratch, int nx, int ny,
                      double dx, int pre, zb_stream_t stream);

/* Training state (device pointers).  Patches: batch images of n x n cells
 * with their own face coefficients cx (batch, n+1, n) and cy (batch, n, n+1)
 * and Dirichlet boundaries.  Residual loss = mean over the batch of
 * |r - A S(r)|^2 / |r|^2, the residual left after one smoother application;
 * see zb_unet_backward for the energy-norm loss.  Adam skips non-finite
 * gradient entries. */
typedef struct {
  int32_t c1, c2, batch, n;
  float cmax;
  float* w_master;        /* float32 master weights                          */
  float* b_master;        /* float32 biases                                  */
  float *m_w, *v_w, *m_b, *v_b;   /* Adam moments                            */
  float *g_w, *g_b;       /* gradients                                       */
  void* w_bf16;           /* bf16 weights used by the forward                */
  void* b_shadow;         /* bf16 scratch for the bias update (>= n_biases)  */
  void* act;              /* >= zb_unet_train_workspace_bytes(c1, c2, batch, n) */
} zb_unet_trainer;

size_t zb_unet_train_workspace_bytes(int c1, int c2, int batch, int n);

/* y = S(r) for the batch (forward only, activations kept for backward). */
int zb_unet_forward(const zb_unet_trainer* t, const float* r, const float* cx,
                    const float* cy, double dx, float* y, zb_stream_t stream);

/* Loss (into *loss_out, device float64, may be NULL) and its gradient with
 * respect to the bf16 weights and the biases into g_w, g_b.  target NULL:
 * the residual loss above; target = the exact errors e (A e = r, same shape as
 * r): the energy-norm loss mean_b (d . A d) / (e . A e), d = e - S(r), the
 * error left after the correction measured as conjugate gradients measure it.
 * Images without signal (denominator <= 1e-30) are left out. */
int zb_unet_backward(const zb_unet_trainer* t, const float* r,
                     const float* target, const float* cx, const float* cy,
                     double dx, double* loss_out, zb_stream_t stream);

/* One Adam step (lr, beta1 0.9, beta2 0.999, eps 1e-8; step counts from 1);
 * refreshes the bf16 weights from the float32 master. */
int zb_unet_adam(const zb_unet_trainer* t, float lr, int step, zb_stream_t stream);

/* Preconditioners of the flexible CG: none (plain CG), the multigrid
 * V-cycle, the V-cycle followed by one learned smoothing step on the finest
 * level (x += S(r - A x), the learned post-smoother), or the V-cycle with the
 * finest level's red-black sweeps replaced by the learned smoother. */
enum { ZB_PRECOND_NONE = 0, ZB_PRECOND_MG = 1, ZB_PRECOND_LEARNED = 2,
       ZB_PRECOND_LEARNED_REPLACE = 3 };

size_t zb_poisson_workspace_bytes(const zb_poisson_cfg* cfg);

/* Byte offsets inside the workspace: [0] r, [1] -1 (z = M r is not kept in
 * float64: [5] is z, converted exactly where it is read), [2] p, [3] q
 * (float64 Krylov vectors), [4] scalars (float64: b.b, r.r, p.q, p.r, z.q,
 * alpha, beta, relative residual at index 7, iteration count at 8), [5] the
 * float32 result of the last V-cycle on level 0 (z = M r), [6] level-0 float32 f, [7]
 * number of levels, [8] first one-CTA level, [9] level-0 float32 x-face
 * coefficients, [10] y-face coefficients.  out holds 11. */
int zb_poisson_layout(const zb_poisson_cfg* cfg, int64_t* out);

/* Face coefficients of every level from the depth h (C values, dtype). */
int zb_poisson_setup(const zb_poisson_cfg* cfg, const void* h, int dtype,
                     void* ws, size_t ws_bytes, zb_stream_t stream);

/* q = A p (float64). */
int zb_poisson_apply(const zb_poisson_cfg* cfg, void* ws, const double* p,
                     double* q, zb_stream_t stream);

/* z = M r: one V-cycle from zero (float32); precond ZB_PRECOND_*. */
int zb_poisson_vcycle(const zb_poisson_cfg* cfg, void* ws, const float* r,
                      float* z, int precond, const zb_smoother* smoother,
                      zb_stream_t stream);

/* b = -div(q*) / dt from the state Q (4, C) (face-averaged fluxes, walls). */
int zb_poisson_rhs(const zb_poisson_cfg* cfg, const void* Q, int dtype,
                   double dt, double* b, zb_stream_t stream);

/* q -= dt * cell-averaged c_f grad p on the momentum rows of Q. */
int zb_poisson_correct(const zb_poisson_cfg* cfg, void* ws, void* Q, int dtype,
                       const double* p, double dt, zb_stream_t stream);

/* Flexible CG (one-term, Notay): start computes r = b - A x, |b|, the first
 * preconditioned direction; each iterate performs one iteration and leaves
 * the relative residual |r| / |b| at scalar index 7.  Both are
 * graph-capturable (no host sync, no allocation). */
int zb_fcg_start(const zb_poisson_cfg* cfg, void* ws, const double* b,
                 double* x, int precond, const zb_smoother* smoother,
                 zb_stream_t stream);
int zb_fcg_iterate(const zb_poisson_cfg* cfg, void* ws, double* x, int precond,
                   const zb_smoother* smoother, zb_stream_t stream);

/* The whole solve as one CUDA graph (start + a conditional WHILE node over
 * iterate): each launch runs from the current x until |r|/|b| <= tol or maxit
 * iterations, without a host round trip; the iteration count is left at
 * scalar index 8.  b, x, ws and the smoother are bound at creation.  Replaces
 * the host GMRES loop of the reference's pressure step
 * (zoomy_jax/fvm/solver_chorin_vam_jax.py:800-823). */
typedef struct zb_fcg_graph zb_fcg_graph;
int zb_fcg_graph_create(const zb_poisson_cfg* cfg, void* ws, const double* b,
                        double* x, int precond, const zb_smoother* smoother,
                        double tol, int maxit, zb_fcg_graph** out,
                        zb_stream_t stream);
int zb_fcg_graph_launch(zb_fcg_graph* graph, zb_stream_t stream);
void zb_fcg_graph_destroy(zb_fcg_graph* graph);

/* Synchronous solve for C callers (the shape of the reference's
 * `jax_gmres(matvec, -b, tol, maxiter)` call plus its residual read-back):
 * FCG from the x given until |r|/|b| <= tol or maxit iterations, one stream
 * synchronisation per iteration; iterations and the final relative residual
 * go to out_iters / out_rel (either may be NULL).  Returns ZB_OK, or
 * ZB_E_NOT_CONVERGED when the tolerance was missed. */
int zb_poisson_solve(const zb_poisson_cfg* cfg, void* ws, const double* b,
                     double* x, double tol, int maxit, int precond,
                     const zb_smoother* smoother, int* out_iters,
                     double* out_rel, zb_stream_t stream);

/* ── unstructured triangles ─────────────────────────────────────────────── */

/* Scheme of the triangle path (the Cartesian fields it shares keep their
 * meaning; limiter: minmod / Barth-Jespersen / none). */
typedef struct {
  int32_t order, recon, riemann, limiter;
  double g, wet_dry_eps, eps_wet, manning_n;
  int32_t implicit_source, dim_factor;
  double cfl, dt_max, t_end;
  int32_t degree, dtype;
} zb_tri_cfg;

/* Device arrays of a triangle mesh (caller-owned; SoA, int32 connectivity,
 * geometry in the state precision except face_inr which is float64).
 * [3][C] arrays hold the cell's three slots plane by plane.  Built by the
 * host from MeshJAX-equivalent data (zoomy_jax/mesh/mesh.py:123-264,
 * solver2/context.py:99-163). */
typedef struct {
  int32_t n_cells, n_faces, n_bf;
  const int32_t* lsq_idx;     /* [3][C] neighbour cell or -1 - boundary face  */
  const void* lsq_wx;         /* [3][C] least-squares weights, x-derivative   */
  const void* lsq_wy;         /* [3][C] least-squares weights, y-derivative   */
  const void* cf_rx;          /* [3][C] face centre - cell centre, x          */
  const void* cf_ry;          /* [3][C] face centre - cell centre, y          */
  const int32_t* cell_face;   /* [3][C] 2 f + side (0 owner, 1 neighbour)     */
  const void* cell_inv_area;  /* [C]                                          */
  const int32_t* face_a;      /* [F] owner cell                               */
  const int32_t* face_b;      /* [F] neighbour cell, or -1 - boundary face    */
  const void* face_nx;        /* [F] unit normal out of the owner             */
  const void* face_ny;
  const void* face_len;       /* [F] face length                              */
  const void* face_rax;       /* [F] face centre - owner centre               */
  const void* face_ray;
  const void* face_rbx;       /* [F] face centre - neighbour centre           */
  const void* face_rby;
  const double* face_inr;     /* [F] min inradius of the two cells (CFL)     */
  const int32_t* bf_kind;     /* [n_bf] ZB_BC_EXTRAPOLATION / ZB_BC_WALL      */
  const void* bf_nx;          /* [n_bf] boundary normals                      */
  const void* bf_ny;
} zb_tri_mesh;

/* Workspace of zb_tri_step / zb_tri_stage / zb_tri_dt. */
size_t zb_tri_workspace_bytes(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh);

/* Control-block set-up for a triangle march from time t0 (the dt slots hold a
 * running minimum of the per-face CFL limit here). */
int zb_tri_init(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh, zb_ctrl* ctrl,
                int phase, double t0, zb_stream_t stream);

/* One full step in place on Q (4, C): the face pass of the first stage
 * reduces the CFL dt over faces (zoomy_jax/fvm/solver2/blocks.py:36-95),
 * SSP-RK2 with gradient / face / gather-update launches per stage
 * (solver_jax.py:722-1131), Manning friction after the step.  Every face is
 * evaluated once and each cell gathers its faces in a fixed order, so the
 * update is deterministic and exactly conservative. */
int zb_tri_step(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh, void* Q,
                void* workspace, size_t workspace_bytes, zb_ctrl* ctrl,
                int phase, zb_stream_t stream);

/* One Shu-Osher stage with a host dt (dt < 0: ctrl->dt), as zb_swe2d_stage. */
int zb_tri_stage(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh,
                 const void* Qk, const void* Q0, void* Q_out, double alpha,
                 double beta, double dt, const void* hinv_src,
                 const uint8_t* force_o1, uint8_t* trouble_out, void* workspace,
                 size_t workspace_bytes, zb_ctrl* ctrl, zb_stream_t stream);

/* dt of the state (CFL law over faces, dt_max, t_end - t) into ctrl->dt. */
int zb_tri_dt(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh, const void* Q,
              void* workspace, size_t workspace_bytes, zb_ctrl* ctrl, double t,
              zb_stream_t stream);

/* Manning source step Q += dt S(Q, hinv0), as zb_swe2d_source. */
int zb_tri_source(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh, void* Q,
                  const void* hinv0, double dt, zb_stream_t stream);

/* Post-step aux rows into Qaux (7, C), as zb_swe2d_aux
 * (zoomy_jax/fvm/solver_jax.py:284-369). */
int zb_tri_aux(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh, const void* Q,
               void* Qaux, zb_stream_t stream);

/* sum h |cell| in float64 into ctrl->mass; partial holds
 * zb_tri_mass_partials() doubles. */
size_t zb_tri_mass_partials(void);
int zb_tri_mass(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh, const void* Q,
                double* partial, zb_ctrl* ctrl, zb_stream_t stream);

/* ── triangle mesh preparation on the GPU ─────────────────────────────────
 * Replaces the host conversion LSQMesh -> MeshJAX (zoomy_jax/mesh/mesh.py:
 * 123-264) and prepare_mesh's index sets (zoomy_jax/fvm/solver2/context.py:
 * 99-163): faces from matched half-edges, owner / neighbour, interior /
 * boundary split, normals, lengths, centre offsets, inradius, least-squares
 * stencils and weights, boundary kinds.  P: [n_vert][2] float64 vertices,
 * T: [n_cells][3] int32 triangles (either orientation; cell order kept), both
 * device pointers.  Face numbers follow (owner cell, local edge), the owner
 * of a shared edge being the lower cell index; boundary faces are numbered in
 * face order. */

/* Scratch bytes of zb_trimesh_match / zb_trimesh_fill (0: too many cells). */
size_t zb_trimesh_scratch_bytes(int32_t n_cells);

/* Phase 1: orient, match the half-edges, number the faces.  Writes the face
 * and boundary-face counts to *n_faces / *n_bf (one stream synchronisation).
 * ZB_E_ARG for a vertex index out of range, a zero-area triangle or an edge
 * shared by more than two triangles. */
int zb_trimesh_match(const double* P, int32_t n_vert, const int32_t* T,
                     int32_t n_cells, void* scratch, size_t scratch_bytes,
                     int32_t* n_faces, int32_t* n_bf, zb_stream_t stream);

/* Phase 2: write the arrays of *mesh (allocated by the caller with the counts
 * of phase 1, geometry in dtype ZB_F32 / ZB_F64, face_inr float64; the
 * pointers are written through).  bc_kind_by_side: 4 host ints, the ZB_BC_*
 * of the left, right, bottom and top sides (a boundary face takes the side
 * its outward normal faces). */
int zb_trimesh_fill(const double* P, int32_t n_cells, const int32_t* bc_kind_by_side,
                    int32_t dtype, const void* scratch, size_t scratch_bytes,
                    zb_tri_mesh* mesh, zb_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* ZB_H */
