/*
 * xac.h — C ABI of libxac.so, the B200 (sm_100a) coupled fluid + thermal
 * lattice-Boltzmann solver that drops in for tgautam03/xAdvCool's solver path.
 *
 * Plain C: pointers, sizes, ints and doubles only. Streams are passed as
 * `void*` holding a cudaStream_t (NULL = the legacy default stream). Every
 * function returns an int status (XAC_OK on success); on failure
 * xac_last_error() returns a message for the calling thread. No C++ exception
 * crosses this boundary.
 *
 * Layouts seen by callers are the reference's:
 *   scalar fields  [nx][ny][nz]        float32, z fastest (wp.array3d)
 *   velocity       [nx][ny][nz][3]     float32 (wp.array3d of vec3f)
 *   populations    [19][nx][ny][nz]    float32 (wp.array4d)
 *   mask           [nx][ny][nz]        int32, values XAC_BC_*
 * The D3Q19 direction order, weights and opposite map are the reference's
 * (src/fluid_engine3d.py:11-53).
 */
#ifndef XAC_H
#define XAC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define XAC_OK 0
#define XAC_EINVAL 1     /* bad argument (null pointer, bad size, bad enum)        */
#define XAC_ECUDA 2      /* a CUDA runtime call failed                             */
#define XAC_EDIVERGED 3  /* the divergence guard fired (NaN, |u|>0.17, T>1e4)      */
#define XAC_ETIMEOUT 4   /* a bounded device-side wait gave up                     */
#define XAC_ENOMEM 5     /* device allocation failed                               */

/* ---- cell labels: src/fluid_engine3d.py:11-14 / src/geometry.py:9-12 ------ */
#define XAC_BC_FLUID 0
#define XAC_BC_SOLID 1
#define XAC_BC_INLET 2
#define XAC_BC_OUTLET 3

/* ---- population storage precision of a lattice ---------------------------- */
/* Population storage; every mode computes in float32. The 16-bit forms store deviations from the rest equilibrium
 * (w_i for the fluid, w_i * T_inlet for the thermal lattice). bfloat16 is used for fluid populations only: a thermal
 * population's deviation is dominated by its advective part w_i*T*3(e_i.u), below which the temperature rise must be
 * resolved. Accuracy (config C3: finned plate, heat power 1e-4, 2000 steps; relative error vs FP64): FP32 R_th and
 * Nu 0.4%; XAC_FP16 R_th 6.2%, Nu 4.1%; XAC_BF16 R_th 10.7%, Nu 9.3%; XAC_FP32_T16 R_th 28%, Nu 21% (a temperature
 * rise of 1e-3 K is below what FP16 resolves next to the advective part). With stronger heating (a 150 x 12 x 8
 * gyroid at heat power 0.05, 300 steps) every 16-bit mode keeps T - T_inlet within 0.2% of FP32 storage (relative
 * L2). */
#define XAC_FP32 0      /* float32 populations in both lattices                                   */
#define XAC_FP16 1      /* binary16 fluid and thermal populations                                 */
#define XAC_BF16 2      /* bfloat16 fluid populations, binary16 thermal populations               */
#define XAC_FP32_T16 3  /* float32 fluid populations, binary16 thermal populations                */

/* ---- stats vector (xac_stats): src/fluid_engine3d.py:283 index order, then
 *      src/thermal_engine3d.py:228 order, then one extra slot ---------------- */
#define XAC_ST_MAX_V 0
#define XAC_ST_SUM_V 1
#define XAC_ST_SUM_KE 2       /* sum of |u|^2 over ALL cells (no 1/2), fluid_engine3d.py:292 */
#define XAC_ST_COUNT 3
#define XAC_ST_SUM_RHO 4
#define XAC_ST_SUM_RHO_IN 5   /* plane x = 1 */
#define XAC_ST_SUM_RHO_OUT 6  /* plane x = nx-2 */
#define XAC_ST_SUM_UX_OUT 7   /* outlet cells */
#define XAC_ST_C_IN 8
#define XAC_ST_C_OUT 9
#define XAC_ST_C_OUTLET 10
#define XAC_ST_MAX_T 11
#define XAC_ST_SUM_T 12
#define XAC_ST_COUNT_T 13
#define XAC_ST_Q_OUT 14       /* sum of u_x*T over outlet cells */
#define XAC_ST_Q_OUT_COUNT 15
#define XAC_ST_NONFINITE 16   /* cells whose |u| or T is not finite */
#define XAC_NSTATS 17

/* ---- scalar outputs (xac_scalars): generate_dataset.py:57-179 plus the
 *      Parquet-only quantities of generate_dataset.py:538-579 ------------------ */
#define XAC_SC_DP 0                /* delta_P over non-solid cells, :99-108        */
#define XAC_SC_RTH 1               /* R_th, :113-140                               */
#define XAC_SC_NU 2                /* Nu, :145-155                                 */
#define XAC_SC_F_FRICTION 3
#define XAC_SC_P_PUMP 4
#define XAC_SC_COP 5
#define XAC_SC_Q_VOL 6
#define XAC_SC_T_MAX_SURFACE 7
#define XAC_SC_T_AVG_SURFACE 8
#define XAC_SC_DELTA_T_MAX 9
#define XAC_SC_SIGMA_T 10
#define XAC_SC_FLUID_TEMP_RISE 11
#define XAC_SC_PRESSURE_DROP_ALL 12  /* Parquet column pressure_drop: all cells of the planes, :556 */
#define XAC_SC_MAX_VELOCITY 13
#define XAC_SC_MAX_TEMPERATURE 14
#define XAC_SC_MEAN_TEMPERATURE 15
#define XAC_SC_DH 16               /* compute_hydraulic_diameter, :57-68           */
#define XAC_SC_V_FLUID 17
#define XAC_SC_A_WETTED 18
#define XAC_SC_POROSITY 19         /* compute_porosity, :71-74                     */
#define XAC_SC_Q_ABSORBED 20       /* intermediate of R_th / Nu, :133-136          */
#define XAC_SC_DT_CONV 21          /* T_avg_surface - T_fluid_avg, :148            */
#define XAC_SC_RHO_AVG 22          /* intermediate of f_friction, :160             */
#define XAC_NSCALARS 23

const char *xac_last_error(void);
int xac_version(void);

/* ========================================================================== *
 * Unfused per-operator entry points, reference layout, caller-owned DEVICE
 * pointers, launched on `stream`. Each replaces one Warp kernel launch
 * (wp.launch(kernel, dim=(nx,ny,nz), inputs=[...])) with the same inputs.
 * ========================================================================== */

/* src/fluid_engine3d.py:58-80 compute_equilibrium_kernel(rho, u, f_eq) */
int xac_equilibrium(const float *rho, const float *u, float *f_eq, int nx, int ny, int nz, void *stream);
/* src/fluid_engine3d.py:85-113 compute_macroscopic_kernel(f, rho, u) */
int xac_macroscopic(const float *f, float *rho, float *u, int nx, int ny, int nz, void *stream);
/* src/fluid_engine3d.py:118-136 bgk_collision_kernel(f_old, f_eq, f_post, mask, tau) */
int xac_bgk_collision(const float *f_old, const float *f_eq, float *f_post, const int32_t *mask, float tau,
                      int nx, int ny, int nz, void *stream);
/* src/fluid_engine3d.py:141-176 fused_equilibrium_collision_kernel(f_old, rho, u, f_post, mask, tau) */
int xac_fused_collision(const float *f_old, const float *rho, const float *u, float *f_post, const int32_t *mask,
                        float tau, int nx, int ny, int nz, void *stream);
/* src/fluid_engine3d.py:181-272 streaming_kernel(f_post, f_streamed, mask, u_inlet[1], rho_outlet, nx, ny, nz);
 * u_inlet is a device pointer to one float, read inside the kernel as the reference does. */
int xac_stream(const float *f_post, float *f_streamed, const int32_t *mask, const float *u_inlet, float rho_outlet,
               int nx, int ny, int nz, void *stream);
/* src/fluid_engine3d.py:277-312 compute_stats_kernel + src/thermal_engine3d.py:226-243 compute_thermal_stats_kernel,
 * merged and made deterministic (FP64 block reductions, fixed combine order). out_host receives XAC_NSTATS doubles;
 * the call synchronises `stream`. */
int xac_stats_fields(const float *rho, const float *u, const float *T, const int32_t *mask, int nx, int ny, int nz,
                     double *out_host, void *stream);
/* No counterpart in the reference. The same stats as xac_stats_fields for callers that cannot allocate device or
 * pinned memory (code running inside a stream capture, or under a memory budget owned by another allocator):
 * it calls no allocator. Its scratch is a fixed 278 KB array in the library's device image, held by every GPU
 * that loads the library; lattices above 2,097,152 cells are rejected (XAC_EINVAL). The result (XAC_NSTATS
 * doubles) goes to the caller's DEVICE buffer out_dev, asynchronously on `stream`. All calls on a device share
 * the scratch, so calls whose GPU work overlaps race. The first call on a device looks up the scratch address;
 * make it before any stream capture. The address is kept for the life of the process: after cudaDeviceReset
 * (which discards the device's copy of the library's module) this entry point must not be called again in that
 * process. */
int xac_stats_fields_noalloc(const float *rho, const float *u, const float *T, const int32_t *mask, int nx, int ny,
                             int nz, double *out_dev, void *stream);

/* src/thermal_engine3d.py:7-47 compute_thermal_equilibrium_kernel(rho, u, T, g_eq, mask) (rho unused, as there) */
int xac_thermal_equilibrium(const float *u, const float *T, float *g_eq, const int32_t *mask, int nx, int ny, int nz,
                            void *stream);
/* src/thermal_engine3d.py:49-86 thermal_bgk_collision_kernel(g_old, g_eq, g_new, mask, tau_f, tau_s, hs, power) */
int xac_thermal_bgk_collision(const float *g_old, const float *g_eq, float *g_new, const int32_t *mask,
                              float tau_fluid, float tau_solid, const float *heat_source, float heat_power, int nx,
                              int ny, int nz, void *stream);
/* src/thermal_engine3d.py:91-145 fused_thermal_equilibrium_collision_kernel(g_old, u, T, g_new, mask, ...) */
int xac_fused_thermal_collision(const float *g_old, const float *u, const float *T, float *g_new,
                                const int32_t *mask, float tau_fluid, float tau_solid, const float *heat_source,
                                float heat_power, int nx, int ny, int nz, void *stream);
/* src/thermal_engine3d.py:147-211 thermal_streaming_kernel(g_post, g_streamed, mask, T_inlet, nx, ny, nz) */
int xac_thermal_stream(const float *g_post, float *g_streamed, const int32_t *mask, float T_inlet, int nx, int ny,
                       int nz, void *stream);
/* src/thermal_engine3d.py:214-224 compute_thermal_macroscopic_kernel(g, T) */
int xac_thermal_macroscopic(const float *g, float *T, int nx, int ny, int nz, void *stream);

/* Test-only operators of validate_analytical.py (kept off the product path). */
/* validate_analytical.py:21-30 dirichlet_thermal_bc_kernel(g, T_val, x_plane, ny, nz) */
int xac_test_dirichlet_plane(float *g, float T_val, int x_plane, int nx, int ny, int nz, void *stream);
/* Test-only: makes the library's bounded waits run out on purpose (an mbarrier that nothing arrives on, as in
 * the staged step kernel; the batched kernel's grid barrier with a block that never arrives), each after `limit`
 * polls (1..2^20). status_out: bit 0 the mbarrier wait gave up, bit 1 the grid barrier gave up, bit 2 the grid
 * barrier recorded XAC_ETIMEOUT; 7 when every wait reported. The context stays usable. */
int xac_test_bounded_waits(unsigned limit, unsigned *status_out, void *stream);
/* Test-only: the convolution kernels' mbarrier wait on a barrier nothing completes, limited to `limit` polls
 * (1..2^20); it must set bit 0 of the flags xac_conv3d_status returns. */
int xac_test_conv_wait_timeout(unsigned limit, void *stream);
/* validate_analytical.py:255-273 periodic_streaming_kernel and :607-621 periodic_thermal_streaming_kernel */
int xac_test_periodic_stream(const float *f_post, float *f_streamed, int nx, int ny, int nz, void *stream);
/* validate_analytical.py:377-395 forced_bgk_collision_kernel(f_old, f_eq, f_new, mask, tau, force_x) */
int xac_test_forced_bgk(const float *f_old, const float *f_eq, float *f_new, const int32_t *mask, float tau,
                        float force_x, int nx, int ny, int nz, void *stream);
/* validate_analytical.py:397-420 periodic_streaming_with_solids_kernel(f_post, f_streamed, mask, nx, ny, nz) */
int xac_test_periodic_stream_solids(const float *f_post, float *f_streamed, const int32_t *mask, int nx, int ny,
                                    int nz, void *stream);
/* validate_analytical.py:502-538 couette_streaming_kernel(f_post, f_streamed, mask, u_wall_x, nx, ny, nz) */
int xac_test_couette_stream(const float *f_post, float *f_streamed, const int32_t *mask, float u_wall_x, int nx,
                            int ny, int nz, void *stream);

/* ========================================================================== *
 * Lattice object: the fused coupled step behind src/simulation.py:14-162.
 * The library owns the population buffers; caller pointers are borrowed for
 * the duration of a call. One lattice per stream; calls on different
 * lattices are thread-safe.
 * ========================================================================== */
typedef struct xac_lattice xac_lattice;

typedef struct xac_desc {
    int nx, ny, nz;
    const int32_t *mask;       /* HOST, [nx][ny][nz], XAC_BC_* labels (simulation.py:65)                    */
    const float *heat_source;  /* HOST, [nx][ny][nz] or NULL = 1 on the z=0 plane; normalised to max 1 here
                                  (simulation.py:77-86)                                                       */
    double tau_fluid;          /* fluid relaxation time                                                      */
    double Pr, k_ratio;        /* thermal taus derived as simulation.py:70-71                                */
    double u_inlet;            /* inlet velocity u_x (simulation.py:62)                                      */
    double rho_outlet;         /* outlet density (simulation.py:61, 1.0)                                     */
    double t_inlet;            /* inlet temperature and cold-start T (simulation.py:73)                      */
    double heat_power;         /* multiplies the normalised heat source (thermal_engine3d.py:117)            */
    int precision;             /* XAC_FP32 / XAC_FP16 / XAC_BF16 / XAC_FP32_T16                               */
} xac_desc;

/* FP64 oracle on the GPU for the reduced-precision storage forms: src/simulation.py:60-100 (heat map normalised in
 * float32, taus derived in double, cold start, then `steps` replays of the six-kernel step) with the unfused
 * reference-layout operators of this library instantiated in double. Fixed step count, no convergence test.
 * desc->mask / heat_source are HOST arrays as for xac_lattice_create (precision ignored); rho [nx][ny][nz],
 * u [nx][ny][nz][3] and T [nx][ny][nz] are DEVICE double buffers, any may be NULL. Allocates its own state. */
int xac_reference_run_fp64(const xac_desc *desc, int steps, double *rho, double *u, double *T, void *stream);

/* simulation.py:60-90: allocate, derive taus, normalise the heat map, cold-start equilibrium. */
int xac_lattice_create(const xac_desc *desc, xac_lattice **out, void *stream);
int xac_lattice_destroy(xac_lattice *lat);
/* Restart from fields (reference layout, DEVICE pointers, any may be NULL = cold-start value): populations are
 * set to the equilibria of (rho, u) and (T, u) exactly as simulation.py:89-90 does for the cold start; solid
 * cells always get rho=1, u=0. This is the warm-start initialiser. */
int xac_lattice_init_fields(xac_lattice *lat, const float *rho, const float *u, const float *T, void *stream);
/* Advance n coupled steps; each equals one replay of the reference's 6-kernel graph (simulation.py:93-100). */
int xac_lattice_step(xac_lattice *lat, int n, void *stream);
/* Stats of the current step (same quantities as simulation.py:124-129), FP64, deterministic; synchronises. */
int xac_lattice_stats(xac_lattice *lat, double out_host[XAC_NSTATS], void *stream);
/* Current macroscopic fields into caller DEVICE buffers, reference layout; any pointer may be NULL. */
int xac_lattice_fields(xac_lattice *lat, float *rho, float *u, float *T, void *stream);
/* Inlet velocity as seen by the streaming step (simulation.py:62, :146 for the pump controller). */
int xac_lattice_set_inlet(xac_lattice *lat, double u_inlet, void *stream);
int xac_lattice_get_inlet(xac_lattice *lat, double *u_inlet, void *stream);
int xac_lattice_steps_done(const xac_lattice *lat, long long *steps);
/* Launch shape of the fused step kernel: threads per block (64, 128, 256) and the visiting order:
 * variant 0 = one thread per row position, in memory order; variant 1 = one block per row whose thermal input is
 * staged in shared memory by bulk copies while the fluid lattice runs (row lengths 64..256; other lengths run
 * variant 0). Variant 1 waits for its copies with a bounded wait; if a wait ever gives up, the call that sees it
 * (xac_lattice_stats, xac_lattice_run) returns XAC_ETIMEOUT and the lattice refuses every further step, run, stats,
 * fields, scalars, validate and save-state call with XAC_ETIMEOUT until xac_lattice_init_fields or
 * xac_lattice_load_state rewrites its populations. Results do not depend on the shape (every cell runs the same
 * arithmetic); xadvcool_b200.autotune picks it. */
int xac_lattice_tune(xac_lattice *lat, int block, int variant);
int xac_lattice_get_tune(const xac_lattice *lat, int *block, int *variant);
/* Diagnostic, no reference counterpart: the floor that the fused step's memory access pattern sets for this
 * lattice. Times `launches` launches of a kernel with the step's threads (the lattice's block size, one thread per
 * row position, the alternating sweep), link-word and slot-table reads, population addresses (fluid pulls of the
 * non-solid cells with the bounce-back reads, thermal pulls, thermal padding fills) and no arithmetic: each value
 * read is stored unchanged. CUDA events on `stream`, after 4 untimed launches. The copies are not a physical state,
 * so the lattice is re-initialised to the cold start (step 0) afterwards. */
int xac_lattice_pattern_copy(xac_lattice *lat, int launches, double *us_per_launch, void *stream);
/* Test hook: writes the lattice's step status word as a staged step kernel whose wait gave up would (no kernel
 * runs), so that a test sees the lattice refuse work and recover after xac_lattice_init_fields. */
int xac_test_set_step_status(xac_lattice *lat, unsigned value, void *stream);
/* Inputs of generate_dataset.py:80 compute_macroscopic_metrics that are not fields. */
typedef struct xac_scalar_params {
    int buf;            /* inlet/outlet buffer length along x (10, generate_dataset.py:90)            */
    int core_nx;        /* heated core extent (src/geometry.py:15: 128, 128)                          */
    int core_ny;
    double t_inlet;     /* 25.0 (generate_dataset.py:88)                                              */
    double tau_fluid;   /* params["tau_fluid"], for k_fluid (:151-152)                                */
    double Pr;          /* (:80)                                                                      */
    double u_inlet;     /* params["u_inlet_val"], for the friction factor (:159)                      */
} xac_scalar_params;

/* generate_dataset.py:57-179 on the current fields, FP64 on the device; writes XAC_NSCALARS doubles and
 * synchronises `stream`. */
int xac_lattice_scalars(xac_lattice *lat, const xac_scalar_params *params, double out_host[XAC_NSCALARS],
                        void *stream);
/* The same on caller fields (reference layout, DEVICE pointers; mask int32). */
int xac_scalars_fields(const float *rho, const float *u, const float *T, const int32_t *mask, int nx, int ny, int nz,
                       const xac_scalar_params *params, double out_host[XAC_NSCALARS], void *stream);
/* Raw population state for checkpoint / restart. */
/* Physical validators of the current fields (analyze_dataset.py:184-323) as FP64 device reductions; out_host
 * receives XAC_NVALIDATE raw values in the order of the XAC_VAL_* slots below, from which
 * xadvcool_b200.validate forms the reference's checks (mass and energy balance, Mach, density deviation,
 * temperature lower bound, pressure-drop sign, divergence). */
#define XAC_VAL_MDOT_IN 0     /* sum rho*ux, non-solid cells of plane x = 1 */
#define XAC_VAL_MDOT_OUT 1    /* the same, plane x = nx-2 */
#define XAC_VAL_MAXV 2        /* max |u| over non-solid cells */
#define XAC_VAL_RHODEV 3      /* max |rho - 1| over non-solid cells */
#define XAC_VAL_TMIN 4        /* min T over non-solid cells */
#define XAC_VAL_NFLUID 5
#define XAC_VAL_RHO1_ALL 6    /* sum rho over all cells of plane x = 1 */
#define XAC_VAL_RHO2_ALL 7    /* the same, plane x = nx-2 */
#define XAC_VAL_DIV_SUM 8     /* sum |div u| over non-solid interior cells (central differences) */
#define XAC_VAL_DIV_MAX 9
#define XAC_VAL_DIV_N 10
#define XAC_VAL_QSRC 11       /* sum of the injected heat source (heat_power x normalised map) */
#define XAC_VAL_ADV_IN 12     /* sum ux over inlet cells of plane x = 0 */
#define XAC_VAL_ADV_OUT 13    /* sum ux*T over outlet cells of plane x = nx-1 */
#define XAC_VAL_DIFF_IN 14    /* sum over plane x = 1 of -k (T[1] - T[0]), k = (tau_th - 0.5)/3 of the cell */
#define XAC_VAL_DIFF_OUT 15   /* sum over plane x = nx-2 of -k (T[nx-1] - T[nx-2]) */
#define XAC_NVALIDATE 16
int xac_lattice_validate(xac_lattice *lat, double *out_host, void *stream);

/* The lattice's own restart format: a 64-byte header (tag "XAC2", size, precision, step count, inlet velocity,
 * number of non-solid cells), the fluid populations of the non-solid cells, the thermal populations and the
 * fields rho, u, T. A state loads only into a lattice of the same size, precision and non-solid cell count, that is
 * one made from the same mask. */
int xac_lattice_state_bytes(const xac_lattice *lat, size_t *bytes);
int xac_lattice_save_state(xac_lattice *lat, void *host_dst, size_t bytes, void *stream);
int xac_lattice_load_state(xac_lattice *lat, const void *host_src, size_t bytes, void *stream);

/* The whole run_simulation loop (simulation.py:102-162) in native code. */
typedef struct xac_run_opts {
    int max_steps;        /* 40000 in the reference signature           */
    int stats_every;      /* 100                                        */
    double tol_ke, tol_T; /* relative-rate thresholds                   */
    int constant_power;   /* 0: constant_flow, 1: constant_power pump   */
    double target_power;
    int min_steps;        /* 0: the reference's rule, no convergence before min(0.6 max_steps, max(5000, 2 nx / u_in))
                           * steps (src/simulation.py:102-104); > 0: that many steps instead (warm starts)            */
} xac_run_opts;

typedef struct xac_run_result {
    long long steps;
    int converged, diverged;
    double d_ke, dT_conv, dQ_conv;
    double u_inlet_final;
    double last_stats[XAC_NSTATS];
} xac_run_result;

/* src/simulation.py:102-162: steps, stats every stats_every steps, the relative-rate convergence test, the
 * divergence guard and the constant-power pump. After the first check the remaining whole intervals run as one
 * CUDA graph launch whose conditional while node repeats {stats_every steps, T, stats, decision kernel} (even
 * stats_every >= 8); the decision kernel does the host loop's double arithmetic, so results do not depend on
 * where the loop runs. Blocks until the run ends. */
int xac_lattice_run(xac_lattice *lat, const xac_run_opts *opts, xac_run_result *res, void *stream);

/* ========================================================================== *
 * Warm-start surrogate convolutions: BF16 tensor-core implicit GEMMs (mma.sync m16n8k16), FP32 accumulation.
 * Activations channels-last [N][D][H][W][C] BF16 (DEVICE pointers); weights [taps][Co][Ci] BF16 with
 * taps = 27 (3x3x3, tap = (dz+1)*9 + (dy+1)*3 + (dx+1)) or 1; zero padding; Ci, Co multiples of 16
 * (Ci, Co <= 256). No reference counterpart: the reference's surrogates run through cuDNN
 * (benchmark/models/unet3d.py:11-125).
 * ========================================================================== */
/* out = act(bias + conv(in, w)); activation 0 = none, 1 = GELU; exactly one of out_bf16 / out_f32. The data
 * gradient is this call on d_out with weights w'[26 - tap][ci][co] = w[tap][co][ci]. */
int xac_conv3d_forward(const void *in, int N, int D, int H, int W, int Ci, const void *weight, const float *bias,
                       int Co, int ksize, int activation, void *out_bf16, float *out_f32, void *stream);
/* dw[tap][co][ci] = sum_v d_out[v][co] in[v + off(tap)][ci] (FP32), db[co] = sum_v d_out[v][co] (db may be NULL);
 * partial: xac_conv3d_partial_floats() floats of device scratch. Deterministic (fixed reduction order). */
int xac_conv3d_weight_grad(const void *in, int N, int D, int H, int W, int Ci, const void *d_out, int Co, int ksize,
                           float *partial, float *dw, float *db, void *stream);
int xac_conv3d_partial_floats(int N, int D, int H, int W, int Ci, int Co, int ksize, long long *count);
/* Reads and clears the device-side status of the convolution kernels (synchronises the device): bit 0 set means a
 * bounded wait inside a tensor-core kernel ran out, and that launch left its output unwritten. */
int xac_conv3d_status(int *flags);

/* ========================================================================== *
 * Design generator on the device: the seeded benchmark families of xadvcool_b200.designs (gyroid_design,
 * mixed_design) evaluated per cell. No reference counterpart on the device: the reference builds masks with numpy
 * (src/geometry.py:339-526). The host draws the random parameters and fills the spec.
 * ========================================================================== */
#define XAC_DESIGN_EMPTY 0      /* no solid inside the frame (src/geometry.py:381-383) */
#define XAC_DESIGN_STRAIGHT 1   /* p0 = channel width, p1 = channel count (src/geometry.py:385-434) */
#define XAC_DESIGN_PIN_FIN 2    /* p0 = pin radius, p1 = pitch: two interleaved square lattices of pins */
#define XAC_DESIGN_GYROID 3     /* p0 = cell size L, p1 = threshold t: solid where the TPMS value > t */
#define XAC_DESIGN_SCHWARZ_P 4
#define XAC_DESIGN_SCHWARZ_D 5
#define XAC_DESIGN_BELOW 16     /* with a TPMS family: solid where the value < p1, as generate_mask does
                                   (src/geometry.py:497-503) */
#define XAC_DESIGN_MAX_HOT 8
typedef struct xac_design_spec {
    int nx, ny, nz;       /* lattice, reference layout [nx][ny][nz] */
    int buf;              /* inlet / outlet buffer cells; the core is x in [buf, nx - buf) */
    int family;           /* XAC_DESIGN_* */
    int margin;           /* TPMS: core x cells at each end kept fluid */
    double p0, p1;        /* family parameters (above) */
    int n_hot;            /* Gaussian hotspots of the z = 0 floor map, <= XAC_DESIGN_MAX_HOT */
    double background;    /* floor map background (0.2) */
    double hot[XAC_DESIGN_MAX_HOT][4];  /* cx, cy (core cells), sigma, amplitude */
} xac_design_spec;
/* mask_dev: int32 [nx][ny][nz] BC labels with the reference frame; heat_dev: float32 [nx][ny][nz], the floor map
 * at z = 0 of the core (0 elsewhere). Both DEVICE pointers. */
int xac_design_build(const xac_design_spec *spec, int32_t *mask_dev, float *heat_dev, void *stream);

/* ========================================================================== *
 * Batch: many designs (uneven lattice sizes, one precision) advanced together by ONE persistent cooperative
 * launch per `steps_per_launch` steps (captured in a CUDA graph where the driver allows it). Each design keeps
 * the convergence test and divergence guard of src/simulation.py:123-156, evaluated on the device; converged
 * and diverged designs retire and their share of the GPU goes to the others. No reference counterpart: the
 * reference solves designs one after another (generate_dataset.py:365-436).
 * ========================================================================== */
typedef struct xac_batch xac_batch;
int xac_batch_create(const xac_desc *designs, int n, xac_batch **out, void *stream);
int xac_batch_destroy(xac_batch *batch);
int xac_batch_size(const xac_batch *batch, int *n);
/* The i-th design as a lattice owned by the batch: warm-start it (xac_lattice_init_fields) before a run, read
 * fields / scalars / stats after. Do not destroy it. */
int xac_batch_lattice(xac_batch *batch, int i, xac_lattice **lat);
/* Threads per block (64, 128, 256; also the cells per tile) and steps per persistent launch. */
int xac_batch_tune(xac_batch *batch, int block, int steps_per_launch);
int xac_batch_get_tune(const xac_batch *batch, int *block, int *steps_per_launch);
/* Run every design from step 0 to convergence, divergence or opts->max_steps; results[i] receives design i's
 * outcome. With opts->constant_power the reference's pump controller (simulation.py:139-146) runs inside the
 * persistent kernel on each design's stats, exactly as xac_lattice_run runs it for one lattice. */
int xac_batch_run(xac_batch *batch, const xac_run_opts *opts, xac_run_result *results, void *stream);
/* Persistent launches of this batch so far: from a captured CUDA graph, and direct (cooperative) launches, which
 * are used when the driver cannot capture the cooperative launch and for launches shorter than steps_per_launch. */
int xac_batch_launch_counts(const xac_batch *batch, long long *graph_launches, long long *direct_launches);

/* Open batch: a design sweep (generate_dataset.py:365-436, one solve per design there) as a queue over one
 * persistent kernel. xac_batch_open makes an empty batch of one precision. xac_batch_admit creates a design in a
 * free slot (at most 1024 slots; a released slot is reused); it joins the running batch at the next multiple of
 * opts->stats_every of the batch's step count, from its own step 0, so every design keeps exactly the steps,
 * decisions and bits of its solo xac_lattice_run. xac_batch_advance runs the batch for up to `steps` steps, and
 * returns early after the launch in which designs finish (so that their slots can be refilled) or when no design
 * is left; it reports the designs that finished during the call (converged,
 * diverged, or at opts->max_steps of their own): their slots, outcomes, and the wall seconds of the launches they
 * took part in, shared among the designs of each launch in proportion to their cells. slots / results /
 * gpu_seconds must hold xac_batch_size() entries. A finished design keeps its lattice (xac_batch_lattice: fields,
 * stats, scalars) until xac_batch_release frees its slot and device memory. xac_lattice_footprint gives the
 * device bytes a design will take, for admission under a memory budget; it reads design->mask when given, since
 * fluid populations are stored for the non-solid cells only (without a mask every cell counts). */
int xac_batch_open(int precision, xac_batch **out);
int xac_batch_admit(xac_batch *batch, const xac_desc *design, int *slot, void *stream);
int xac_batch_advance(xac_batch *batch, const xac_run_opts *opts, long long steps, int *n_finished, int *slots,
                      xac_run_result *results, double *gpu_seconds, void *stream);
int xac_batch_release(xac_batch *batch, int slot);
int xac_lattice_footprint(const xac_desc *design, unsigned long long *bytes);

#ifdef __cplusplus
}
#endif
#endif /* XAC_H */
