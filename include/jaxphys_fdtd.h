/*
 * jaxphys_fdtd.h -- C ABI of the B200 (sm_100a) FDTD Maxwell engine.
 *
 * Drop-in boundary for the Yee solvers of jaxphys (package `neurosim`):
 *   3D: src/neurosim/em/fdtd3d.py  (EMGrid3D, PointSource3D, DielectricRegion)
 *   2D: src/neurosim/em/fdtd.py    (EMGrid, PlaneWave, Wall)
 * The reference has no native layer: its Python classes call jax.numpy and
 * jax.lax.scan directly.  Each entry point below replaces the piece of that
 * Python code cited beside it; a host binding (ctypes, cgo, JNI, N-API) needs
 * only plain pointers, sizes and integers.
 *
 * Conventions
 *  - Every function returns JXF_OK (0) or a JXF_ERR_* code; the message of the
 *    last failure on the calling thread is jxf_last_error().
 *  - Fields are float32, C order (nx, ny, nz) / (nx, ny), z (resp. y) fastest,
 *    one array per component: the layout of a NumPy / JAX / torch array of
 *    that shape, so DLPack capsules map 1:1 onto the pointers.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *    All device work is ordered on it; nothing synchronises the host except
 *    the copies to host memory (which synchronise `stream`).
 *  - A handle owns its device memory (ping-pong field buffers, CPML psi slabs,
 *    coefficient tables, source/probe tables).  A handle is not thread safe.
 *  - Component ids: 0..5 = Ex, Ey, Ez, Hx, Hy, Hz (2D: 0..2 = Ez, Hx, Hy).
 */
#ifndef JAXPHYS_FDTD_H
#define JAXPHYS_FDTD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JXF_OK 0
#define JXF_ERR_INVALID 1    /* bad argument / configuration            */
#define JXF_ERR_CUDA 2       /* a CUDA runtime / driver call failed      */
#define JXF_ERR_OOM 3        /* device allocation failed                 */
#define JXF_ERR_TIMEOUT 4    /* a bounded device wait gave up            */
#define JXF_ERR_NONFINITE 5  /* NaN / Inf found by jxf_grid3d_check_finite */

/* Boundary modes.  ABSORBING and PERIODIC are the reference's
 * (fdtd3d.py:94,247-301,361-366; fdtd.py:97,314-352).  PEC is the reference's
 * non-periodic stencil without the damping multiply (what fdtd3d.py does for
 * any boundary string other than the two above).  CPML is an extension:
 * convolutional PML with psi recurrences.  REFLECTING is 2D only
 * (fdtd.py:264-282). */
#define JXF_BND_ABSORBING 0
#define JXF_BND_PERIODIC 1
#define JXF_BND_PEC 2
#define JXF_BND_CPML 3
#define JXF_BND_REFLECTING 4

/* Kernel path selection for 3D grids. */
#define JXF_PATH_AUTO 0      /* TMA path when the shape allows it          */
#define JXF_PATH_GENERIC 1   /* plain-load kernels: every mode and shape   */
#define JXF_PATH_TMA 2       /* TMA-staged marching kernel (nz % 4 == 0,   */
                             /* boundary != PERIODIC)                       */

typedef struct jxf_grid3d jxf_grid3d;
typedef struct jxf_grid2d jxf_grid2d;

/* Replaces EMGrid3D.__init__ (fdtd3d.py:90-105) plus the coefficient set-up
 * of simulate() (fdtd3d.py:185-224: dt, dt/(mu0 dx), dt/(eps0 dx), the PML
 * sigma profile of :139-167 and its damping factor of :363). */
typedef struct {
  int32_t nx, ny, nz;
  double dx;             /* cell size (m)                                   */
  double dt;             /* time step (s); <= 0 selects 0.99 dx/(c sqrt 3)  */
  int32_t boundary;      /* JXF_BND_*                                       */
  int32_t pml_layers;    /* damping layers (ABSORBING) or CPML thickness    */
  double cpml_order;     /* CPML polynomial grading m        (default 3)    */
  double cpml_r0;        /* CPML normal reflection target    (default 1e-6) */
  double cpml_kappa_max; /* CPML kappa_max                   (default 1)    */
  double cpml_alpha_max; /* CPML CFS alpha_max, S/m          (default 0)    */
  int32_t path;          /* JXF_PATH_*                                      */
  int32_t device;        /* CUDA device ordinal                             */
} jxf_grid3d_desc;

typedef struct {
  double dt, coef_h, coef_e;  /* dt, dt/(mu0 dx), dt/(eps0 dx)            */
  int64_t step;               /* steps taken since the last reset         */
  int32_t path;               /* JXF_PATH_GENERIC or JXF_PATH_TMA in use  */
  int32_t tile_z, tile_y, rows_per_thread, stages, x_chunk;
  int64_t device_bytes;       /* device memory held by the handle         */
  int32_t kernels_per_step;   /* step kernels launched per leapfrog step  */
  int32_t shell_blocks, interior_blocks;  /* CPML region split (TMA path) */
  int32_t tma_config;         /* launch-shape registry entry (TMA path)   */
  int32_t axis_split;         /* single-axis CPML shell split on (1)/off  */
  int32_t blocked_config;     /* two-level blocked registry entry, or -1  */
  int32_t blocked_x_chunk;    /* planes per block of the blocked launch   */
  int32_t blocked_kernels_per_pass; /* launches per blocked pass (2 steps) */
} jxf_grid3d_info;

int jxf_grid3d_create(const jxf_grid3d_desc* desc, jxf_grid3d** out);
int jxf_grid3d_destroy(jxf_grid3d* g);
int jxf_grid3d_get_info(const jxf_grid3d* g, jxf_grid3d_info* out);

/* Number of TMA launch shapes in the registry, and a way to pin one: cfg in
 * [0, jxf_num_tma_configs()) and the planes each block marches over;
 * cfg < 0 returns to autotuning (which runs on the first step otherwise). */
int jxf_num_tma_configs(void);
int jxf_grid3d_set_launch(jxf_grid3d* g, int32_t cfg, int32_t x_chunk);
/* CPML grids on the TMA path: on != 0 runs the shell blocks that touch the
 * psi slab of one axis only on kernels specialised for that axis (4 psi
 * arrays instead of 12, smaller shared memory); the autotuner chooses it per
 * grid shape, this pins it (with jxf_grid3d_set_launch). */
int jxf_grid3d_set_axis_split(jxf_grid3d* g, int32_t on);
/* Two-level temporal blocking (TMA path; replaces two iterations of the
 * reference's scan body, fdtd3d.py:280-379, per pass over the fields): cfg in
 * [0, jxf_num_blocked_configs()) advances pairs of steps with one blocked
 * pass each (an odd remainder takes one ordinary step), x_chunk planes per
 * block; cfg < 0 keeps one step per pass.  The autotuner chooses it per grid
 * shape; this pins it. */
int jxf_num_blocked_configs(void);
int jxf_grid3d_set_blocked(jxf_grid3d* g, int32_t cfg, int32_t x_chunk);

/* Relative permittivity, replaces _build_epsilon_r (fdtd3d.py:132-137) and
 * the per-cell factor (dt_eps_dx / eps_r) of fdtd3d.py:299,336,345,354.
 * eps_r: nx*ny*nz float64 values in HOST memory (the library forms
 * dt/(eps0 dx)/eps_r in FP64 and rounds once), or NULL for vacuum.
 * eps_r = +inf (extension) marks a perfect electric conductor cell: its
 * factor is 0, so Ex, Ey and Ez of that cell keep their initial value (zero);
 * zero, negative and NaN values are rejected. */
int jxf_grid3d_set_eps_host(jxf_grid3d* g, const double* eps_r);
/* Same from a DEVICE float32 array (e.g. a DLPack capsule's data pointer):
 * the division runs on the device in FP32 (+inf gives 0, as above). */
int jxf_grid3d_set_eps_device(jxf_grid3d* g, const float* eps_r, void* stream);

/* Soft sources, replaces add_sources (fdtd3d.py:233-245): after the E update
 * (and damping) of step n, E_comp[cell] += amplitude * wave[wave_id][n].
 * Entries with the same cell are applied in list order.  cell is the linear
 * index (ix*ny + iy)*nz + iz, comp in 0..2. */
int jxf_grid3d_set_sources(jxf_grid3d* g, int32_t n, const int64_t* cell,
                           const int32_t* comp, const float* amplitude,
                           const int32_t* wave_id);
/* Waveform samples for absolute steps 0..n_samples-1 of every wave id
 * (row-major [n_waves][n_samples], host memory).  The reference's
 * sin(2 pi f (t0 + n dt)) (fdtd3d.py:238,288) is tabulated by the caller in
 * FP64. */
int jxf_grid3d_set_waveforms(jxf_grid3d* g, int32_t n_waves, int64_t n_samples,
                             const float* samples);

/* Probes (extension): record field comp (0..5) at cell after every step. */
int jxf_grid3d_set_probes(jxf_grid3d* g, int32_t n, const int64_t* cell,
                          const int32_t* comp);

/* Advance n_steps leapfrog steps; replaces one jax.lax.scan over `step`
 * (fdtd3d.py:280-393).  probe_out: DEVICE float32 [n_steps][n_probes] or
 * NULL.  Returns JXF_ERR_TIMEOUT if a bounded device wait gave up (checked
 * only when the call synchronises; see jxf_grid3d_check_error).  An x-slab
 * (jxf_grid3d_create_slab) takes it only on the TMA path, one step per call. */
int jxf_grid3d_step(jxf_grid3d* g, int32_t n_steps, float* probe_out, void* stream);

/* Adjoint (extension; the reference differentiates nothing in its FDTD,
 * and jax.grad through EMGrid3D.simulate, fdtd3d.py:393, would keep every
 * step).  Gradient of an objective J(probe traces) with respect to the
 * per-cell relative permittivity, by the exact transpose of the discrete
 * step, with sqrt(T) checkpointing.
 *
 * jxf_grid3d_adjoint_forward: reset, then run n_steps recording the probes
 * into probe_out (device [n_steps][n_probes], may be NULL) and keeping a
 * checkpoint of the full state every checkpoint_every steps (<= 0:
 * ceil(sqrt(n_steps))).
 * jxf_grid3d_adjoint_backward: probe_grad = dJ/d(probe_out) (device
 * [n_steps][n_probes]); writes dJ/d(eps_r) (device float32 [nx*ny*nz]).
 * Recomputes each segment forward from its checkpoint (one segment of H and
 * psi_E snapshots is held) and runs the adjoint steps in reverse.  Leaves
 * the grid at its initial (step 0) state.  Not for PERIODIC grids. */
int jxf_grid3d_adjoint_forward(jxf_grid3d* g, int32_t n_steps, int32_t checkpoint_every,
                               float* probe_out, void* stream);
int jxf_grid3d_adjoint_backward(jxf_grid3d* g, const float* probe_grad, float* grad_eps,
                                void* stream);

/* Decomposition of one grid along x over several processes (one per GPU;
 * the reference runs a single device).  jxf_grid3d_create_slab makes the
 * handle of global planes [x0, x1) of the grid `desc`, stored with one ghost
 * plane on each side (local plane 0 = global x0-1, local plane x1-x0+1 =
 * global x1).  A step is: fill local plane x1-x0+1 with Ey, Ez of global
 * plane x1 (the next rank's first plane), jxf_grid3d_half_step(H); fill
 * local plane 0 with Hy, Hz of global plane x0-1 (the previous rank's last
 * plane), jxf_grid3d_half_step(E) -- which also applies this rank's sources
 * and records its probes into probe_row.  Sources and probes take LOCAL cell
 * indices.  jxf_grid3d_plane copies one plane of one component between the
 * grid and a device buffer (to_buf != 0: grid -> buffer).  PERIODIC grids are
 * not decomposed.
 *
 * With desc->path == JXF_PATH_TMA (nz % 4 == 0) the slab instead takes whole
 * steps on the one-step TMA kernel, jxf_grid3d_step with n_steps = 1:
 * before each, fill local plane x1-x0+1 with Ey, Ez of global plane x1 and
 * local plane 0 with Ex, Ey, Ez of global plane x0-1 (the neighbours' edge
 * planes of the current state).  The kernel recomputes H on local plane 0 as
 * a bitwise replica of the previous rank's last plane (its psi included) and
 * never updates E on a ghost plane.  Half steps are refused on such slabs. */
int jxf_grid3d_create_slab(const jxf_grid3d_desc* desc, int32_t x0, int32_t x1,
                           jxf_grid3d** out);
int jxf_grid3d_half_step(jxf_grid3d* g, int32_t half, float* probe_row, void* stream);
/* The same half-step in two parts, so the exchange with a neighbour overlaps
 * the bulk of the update: part 1 updates only the plane this half-step hands
 * to a neighbour (H: the last owned plane; E: the first owned plane, with its
 * sources), part 2 the other owned planes (E: with their sources, then the
 * probes; the step counter advances after E part 2).  part 0 = the whole
 * half-step.  Same results as jxf_grid3d_half_step bit for bit.  No reference
 * counterpart (the reference runs on one device). */
int jxf_grid3d_half_step_part(jxf_grid3d* g, int32_t half, int32_t part, float* probe_row,
                              void* stream);
int jxf_grid3d_plane(jxf_grid3d* g, int32_t comp, int32_t plane, float* buf, int32_t to_buf,
                     void* stream);

/* Batches of independent grids (extension; the reference runs one grid per
 * simulate() call).  jxf_batch3d_create groups existing grids (generic path,
 * same boundary mode and device; sizes may differ); they keep their own
 * materials, sources, probes and field access.  jxf_batch3d_step advances
 * every grid by n_steps with one kernel per phase for the whole batch; with
 * use_graph != 0 the n-step sequence is captured once into a CUDA graph
 * (cached per start step and length) and replayed with one launch.  Probe
 * rows of the last run: jxf_batch3d_probes(b, grid, n_steps, dst) copies the
 * [n_steps][n_probes of that grid] trace into device memory. */
typedef struct jxf_batch3d jxf_batch3d;
int jxf_batch3d_create(int32_t n, jxf_grid3d* const* grids, jxf_batch3d** out);
int jxf_batch3d_destroy(jxf_batch3d* b);
int jxf_batch3d_reset(jxf_batch3d* b, void* stream);
int jxf_batch3d_step(jxf_batch3d* b, int32_t n_steps, int32_t use_graph, void* stream);
int jxf_batch3d_probes(jxf_batch3d* b, int32_t grid, int32_t n_steps, float* dst, void* stream);
/* Kernel launches per leapfrog step of the batch's current shape, and the
 * launch shape of a TMA batch (registry entry, x chunk, single-axis split;
 * -1 each for a generic batch).  No reference counterpart (the reference runs
 * one grid per simulate() call, fdtd3d.py:169). */
int jxf_batch3d_kernels_per_step(const jxf_batch3d* b);
int jxf_batch3d_launch(const jxf_batch3d* b, int32_t* out3);

/* Learned absorbing band (extension; the reference has only the graded PML).
 * A jxf_band holds one small network per face of a box (6 faces,
 * f = 2 * axis + side): 54 inputs (the 3 x 3 stencil of Ex..Hz, H scaled by
 * eta0, over the 3 outermost cell layers along the face normal and
 * -1, 0, +1 along its first tangent axis, normalised by their RMS s),
 * 2 hidden layers of 64 (tanh-form GELU), 6 outputs; BF16 weights, FP32
 * accumulation on the tensor cores.  After each plain step of a PEC-walled
 * grid, every cell of the outer layer gets X += s * output (H / eta0).
 * Parameters per face (FP32, JXF_BAND_PARAMS floats): W1[64][64] (out, in;
 * inputs 54..63 zero), b1[64], W2[64][64], b2[64], W3[16][64] (rows 6..15
 * zero), b3[16].
 *   jxf_band_collect   appends training rows for the outer cells of a grid
 *                      given by 6 device field pointers (its state after one
 *                      plain step from a reference state) against the
 *                      reference's next state (6 device pointers of a larger
 *                      grid, the box at offset (ox, oy, oz)); row weight s^2.
 *   jxf_band_grad      gradient and loss (sum of w |out - target|^2 / sum w,
 *                      per face) over the whole dataset, no update.
 *   jxf_band_train     iters Adam steps on batch_rows random rows per face;
 *                      loss[i] (nullable) = summed face losses of step i.
 *   jxf_band_eval      outputs for given normalised feature rows (testing).
 *   jxf_batch3d_set_band / jxf_grid3d_set_band attach a band to a batch of
 *                      PEC grids / to one PEC grid on the generic path (NULL
 *                      detaches); every later step applies it.
 *                      jxf_band_destroy fails (JXF_ERR_INVALID) while a grid
 *                      or batch still has the band attached. */
#define JXF_BAND_PARAMS 9360
#define JXF_BAND_FACES 6
#define JXF_BAND_FEATURES 54
typedef struct jxf_band jxf_band;
int jxf_band_create(int32_t device, jxf_band** out);
int jxf_band_destroy(jxf_band* m);
int jxf_band_set_params(jxf_band* m, const float* params);
int jxf_band_get_params(jxf_band* m, float* params);
int jxf_band_eval(jxf_band* m, int32_t n, const float* feat, const int32_t* face, float* out);
int jxf_band_collect(jxf_band* m, float* const* fields, int32_t nx, int32_t ny, int32_t nz,
                     const float* const* ref, int32_t rnx, int32_t rny, int32_t rnz, int32_t ox,
                     int32_t oy, int32_t oz, void* stream);
int jxf_band_dataset_size(jxf_band* m, int64_t* rows);
int jxf_band_dataset_clear(jxf_band* m);
int jxf_band_dataset_get(jxf_band* m, int32_t face, int64_t first, int64_t count, uint16_t* feat,
                         float* target, float* weight);
int jxf_band_grad(jxf_band* m, float* grad, float* loss, void* stream);
int jxf_band_train(jxf_band* m, int32_t iters, int32_t batch_rows, float lr, uint64_t seed,
                   float* loss, void* stream);
int jxf_band_check_error(jxf_band* m, void* stream);
int jxf_batch3d_set_band(jxf_batch3d* b, jxf_band* m);
int jxf_grid3d_set_band(jxf_grid3d* g, jxf_band* m);

/* Zero fields and psi, reset the step counter. */
int jxf_grid3d_reset(jxf_grid3d* g, void* stream);

/* Device pointer of the CURRENT buffer of component comp (0..5).  Valid until
 * the next jxf_grid3d_step (buffers alternate between steps). */
int jxf_grid3d_field_ptr(jxf_grid3d* g, int32_t comp, float** out);
/* Copy component comp out of / into the grid.  *_is_host selects host or
 * device memory for the other side.  Copies to host synchronise `stream`. */
int jxf_grid3d_get_field(jxf_grid3d* g, int32_t comp, float* dst, int32_t dst_is_host,
                         void* stream);
int jxf_grid3d_set_field(jxf_grid3d* g, int32_t comp, const float* src,
                         int32_t src_is_host, void* stream);
/* Copy all six components into dst (device, 6*nx*ny*nz floats, component
 * major): one saved frame of EMFieldHistory3D (fdtd3d.py:371-417). */
int jxf_grid3d_snapshot(jxf_grid3d* g, float* dst, void* stream);

/* Synchronise `stream` and report a device-side error flag (bounded-wait
 * timeout) raised by earlier steps; clears the flag. */
int jxf_grid3d_check_error(jxf_grid3d* g, void* stream);
/* Synchronise and scan the six fields for NaN/Inf (JXF_ERR_NONFINITE). */
int jxf_grid3d_check_finite(jxf_grid3d* g, void* stream);

/* Allocation-free stepping.  No counterpart in the reference (its solver
 * allocates fresh JAX arrays on every call).  For callers that may not call
 * cudaMalloc: code living inside another framework's device memory pool (an
 * XLA custom call, for instance, which must not take device memory behind
 * the pool's back) or hosts that forbid allocation at run time.  Advances the caller's six float32
 * field buffers (device, C order (nx, ny, nz), Ex..Hz) by n_steps with the
 * reference's ABSORBING or PEC update and no sources, using a fixed device
 * scratch array inside the library (about 6 MB, held by every GPU that loads
 * the library until exit) instead of allocations.  Limit: at most
 * JXF_NOALLOC_MAX_CELLS cells, at most 4096 per axis, nz % 4 == 0; larger
 * grids are rejected with JXF_ERR_INVALID.  cb: device per-cell
 * dt/(eps0 dx eps_r) (float32) or NULL for vacuum.  Every pointer must be
 * 16-byte aligned (JXF_ERR_INVALID otherwise).  The first call on a
 * device resolves the scratch address (cudaGetSymbolAddress), so make it
 * before any stream capture.  All calls share the scratch: calls that
 * overlap on the GPU (other streams, other threads) race.  Synchronises
 * `stream` before returning. */
#define JXF_NOALLOC_MAX_CELLS 262144
typedef struct {
  int32_t nx, ny, nz;
  double dx;
  double dt;          /* <= 0 selects 0.99 dx/(c sqrt 3) */
  int32_t boundary;   /* JXF_BND_ABSORBING or JXF_BND_PEC */
  int32_t pml_layers;
  int32_t device;
} jxf_noalloc_desc;
int jxf_grid3d_run_noalloc(const jxf_noalloc_desc* desc, float* const* fields,
                           const float* cb, int32_t n_steps, void* stream);

/* ---------------------------------------------------------------- 2D (TM) */

/* Replaces EMGrid.__init__ (fdtd.py:93-113) and the set-up part of
 * simulate() (fdtd.py:209-255). */
typedef struct {
  int32_t nx, ny;
  double dx;
  double dt;            /* <= 0 selects 0.99 dx/(c sqrt 2) (fdtd.py:214) */
  int32_t boundary;     /* ABSORBING, PERIODIC or REFLECTING              */
  int32_t pml_layers;
  int32_t device;
} jxf_grid2d_desc;

int jxf_grid2d_create(const jxf_grid2d_desc* desc, jxf_grid2d** out);
int jxf_grid2d_destroy(jxf_grid2d* g);
/* Line sources, replaces fdtd.py:257-262: Ez[:, y] += amp * wave[w][n]. */
int jxf_grid2d_set_sources(jxf_grid2d* g, int32_t n, const int32_t* y,
                           const float* amplitude, const int32_t* wave_id);
int jxf_grid2d_set_waveforms(jxf_grid2d* g, int32_t n_waves, int64_t n_samples,
                             const float* samples);
/* Conductors, replaces _build_conductor_mask (fdtd.py:144-157): row y is
 * PEC except x in [gap_start, gap_end); gap_start < 0 means a solid wall. */
int jxf_grid2d_set_walls(jxf_grid2d* g, int32_t n, const int32_t* y,
                         const int32_t* gap_start, const int32_t* gap_end);
/* Replaces the scan over fdtd.py:304-364. */
int jxf_grid2d_step(jxf_grid2d* g, int32_t n_steps, void* stream);
int jxf_grid2d_reset(jxf_grid2d* g, void* stream);
int jxf_grid2d_field_ptr(jxf_grid2d* g, int32_t comp, float** out);
int jxf_grid2d_get_field(jxf_grid2d* g, int32_t comp, float* dst, int32_t dst_is_host,
                         void* stream);
int jxf_grid2d_set_field(jxf_grid2d* g, int32_t comp, const float* src,
                         int32_t src_is_host, void* stream);
/* Copy Ez, Hx, Hy into dst (device, 3*nx*ny floats): one EMFieldHistory
 * frame (fdtd.py:359-386). */
int jxf_grid2d_snapshot(jxf_grid2d* g, float* dst, void* stream);
int jxf_grid2d_check_error(jxf_grid2d* g, void* stream);

/* ------------------------------------------------------ field viewers */
/* Extension, for the snapshot / animation writers (jaxphys_b200.viz) that
 * replace the reference's matplotlib viewers (viz/fields.py:32-167) and read
 * the fields where they live.  A slice is nu x nv FP32 samples at
 * src[f*sf + c*su + r*sv] (DEVICE memory; strides in elements) for frames
 * f < n_frames.
 *
 * *out (DEVICE float) = max |v| over all frames (stream-ordered). */
int jxf_slice_absmax(const float* src, int64_t nu, int64_t nv, int64_t su, int64_t sv,
                     int32_t n_frames, int64_t sf, float* out, void* stream);
/* out (DEVICE, n_frames * nv * nu * 3 bytes): RGB images as the reference's
 * imshow(data.T, origin="lower", vmin=-vmax, vmax=vmax): image row 0 is slice
 * row nv-1, colour lut[k] (256 RGB entries, DEVICE) with
 * k = floor((v/vmax + 1)/2 * 256) clamped to [0, 255].  vmax is read from
 * vmax_dev when not NULL (e.g. jxf_slice_absmax's output), else the vmax
 * argument; a zero vmax counts as 1 (viz/fields.py:63-65). */
int jxf_slice_rgb(const float* src, int64_t nu, int64_t nv, int64_t su, int64_t sv,
                  int32_t n_frames, int64_t sf, const float* vmax_dev, float vmax,
                  const uint8_t* lut, uint8_t* out, void* stream);

/* ------------------------------------------------------------------ misc */
const char* jxf_last_error(void);
/* Library version (major*10000 + minor*100 + patch). */
int jxf_version(void);

#ifdef __cplusplus
}
#endif

#endif /* JAXPHYS_FDTD_H */
