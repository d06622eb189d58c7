/*
 * ce_gpu.h -- C ABI of the B200 Coulomb-explosion engine (libce_gpu.so).
 *
 * The drop-in boundary for the reference's batched explosion path. The reference
 * exposes that path as a C++ class template (include/coulomb/batched_integrator.hpp);
 * a C++ host (coulomb::gpu::BatchedRK45, host/include/coulomb/gpu/batched_rk45.hpp)
 * or any FFI binds these plain entry points instead:
 *
 *   reference                                                  replaced by
 *   BatchedRK45<T>(mol, coulomb_k, lanes, rtol, atol)          ce_create + ce_set_molecule
 *     include/coulomb/batched_integrator.hpp:71-106
 *   BatchedRK45<T>::set_lane_geometry(lane, pos)               the pos[S][N][3] argument
 *     include/coulomb/batched_integrator.hpp:112-121
 *   BatchedRK45<T>::run(RunConfig) -> Result                   ce_run / ce_run_device
 *     include/coulomb/batched_integrator.hpp:123-191
 *   run_to_convergence(mol, force, integrator, state, cfg)     ce_run (per sim, batched)
 *     src/driver.cpp:7-46
 *
 * Conventions: plain pointers and sizes, no exceptions across the ABI. Every
 * function returns CE_OK (0) or a negative CE_ERR_* code; ce_last_error() gives
 * the message. Per-sim failures are NOT call failures: they are reported in
 * the per-sim status array (CE_SIM_*), mirroring the reference precision
 * sweep's FailureCode (bench/bench_precision_sweep.cpp:80-85).
 *
 * Units: atomic units throughout (Coulomb constant passed explicitly, 1.0 in
 * atomic units); masses in electron masses (amu * 1822.888486209,
 * include/coulomb/units.hpp:11-14). Every simulation starts at rest.
 *
 * Threading: one engine per host thread; calls on one engine are stream-ordered
 * and not thread-safe (the reference's BatchedRK45 likewise holds mutable state).
 */
#ifndef CE_GPU_H
#define CE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- call status ---- */
#define CE_OK 0
#define CE_ERR_INVALID (-1)   /* bad argument: the reference's std::invalid_argument */
#define CE_ERR_CUDA (-2)      /* a CUDA runtime call failed                        */
#define CE_ERR_NO_DEVICE (-3) /* no usable sm_100 device                            */
#define CE_ERR_STATE (-4)     /* engine not ready (no molecule set, ...)            */

/* ---- per-sim status (uint8), bench/bench_precision_sweep.cpp:80-85 ---- */
#define CE_SIM_OK 0           /* reached PE <= pe_stop_fraction * PE_0               */
#define CE_SIM_REJECT_LIMIT 1 /* > 100 rejections in one step (reference throws,
                                 src/integrators.cpp:78-82); state kept as is       */
#define CE_SIM_MAX_STEPS 2    /* max_steps reached first (converged = false,
                                 src/driver.cpp:20-23)                                */
#define CE_SIM_NONFINITE 3    /* non-finite initial potential energy (NaN input)    */
#define CE_SIM_BAD_INPUT 4    /* mixed batches: atom count outside 1..10            */

/* ---- precision mode bits (ce_run_config.precision_mode) ---- */
#define CE_PREC_FP32 0  /* FP32 state, FP32 time and stop test (reference f32 engine)   */
#define CE_PREC_KAHAN 1 /* + compensated (Kahan) accumulation of the x / v updates      */
#define CE_PREC_FP64 2  /* + FP64 time accumulator and FP64-summed stop-test energy     */

#define CE_MAX_ATOMS 10

typedef struct ce_engine ce_engine;

/* RunConfig (include/coulomb/driver.hpp:141-163) + IntegratorOptions
 * (include/coulomb/integrator.hpp:230-233) in one struct. */
typedef struct ce_run_config {
  double rtol;             /* relative tolerance (reference default 1e-8)            */
  double atol;             /* absolute tolerance (reference default 1e-16)           */
  double pe_stop_fraction; /* stop at PE <= f * PE_0 (reference default 1e-9)        */
  double max_dt;           /* step cap (reference default 1e12)                      */
  uint64_t max_steps;      /* accepted-step cap (reference default 1e6)              */
  int32_t redistribute_energy; /* rescale v so KE = E_0 (reference default true)     */
  int32_t precision_mode;  /* CE_PREC_* bits                                         */
} ce_run_config;

/* Fill `cfg` with the reference defaults (driver.hpp:147-162, integrator.hpp:231-232). */
void ce_default_config(ce_run_config* cfg);

/* Per-sim outputs. For ce_run these are host pointers, for ce_run_device device
 * pointers; same layouts. momenta is required, every other field may be NULL.
 *   momenta   [S][N][3] float  m_i v_i after redistribution (Result::momenta,
 *                              batched_integrator.hpp:65, (lane*n+i)*3+c order)
 *   ker       [S] double       sum |p_i|^2 / (2 m_i)  (demo/sanity_check.py:82-83)
 *   steps     [S] uint32       accepted steps (Result::steps)
 *   status    [S] uint8        CE_SIM_*  (Result::converged == (status == 0))
 *   rejects   [S] uint32       rejected attempts over the run
 *   t_final   [S] double       simulated time at termination (RunResult::t_final)
 *   pe_final  [S] double       potential energy at termination (RunResult::pe_final)
 *   ke_before [S] double       kinetic energy before redistribution
 *                              (RunResult::ke_before_redist)
 *   positions [S][N][3] float  positions at termination (the state's positions
 *                              after run_to_convergence, src/driver.cpp:7-46)
 *   e0        [S] double       initial total energy E_0 = PE_0 (RunResult::energy_initial) */
typedef struct ce_outputs {
  float* momenta;
  double* ker;
  uint32_t* steps;
  uint8_t* status;
  uint32_t* rejects;
  double* t_final;
  double* pe_final;
  double* ke_before;
  float* positions;
  double* e0;
} ce_outputs;

/* Launch-shape knobs (0 = autotuned value if any, else the engine default). */
typedef struct ce_tuning {
  int32_t block_threads;    /* threads per block, multiple of 32 up to 256; the     *
                             * lane-per-atom and mixed kernels run at most 128 and  *
                             * clamp a larger request; thread-per-sim runs 128 (64  *
                             * from 8 atoms), two threads per sim 128               */
  int32_t blocks_per_sm;    /* persistent grid = SMs * this (0: occupancy limit)    */
  int32_t refill_threshold; /* refill a warp once this many sims are idle (1..32;   *
                             * 0: a default per molecule size)                       */
  int32_t lanes_per_sim;    /* 1 = one thread per sim; 2 = two threads per sim     *
                             * (3+ atoms; at 2 atoms, one lane per atom); 3..10 =   *
                             * one lane per atom. Mixed batches: 2 = two threads    *
                             * per sim in the per-size schedules (a one-launch      *
                             * request then runs per size), otherwise one lane per  *
                             * atom                                                  */
} ce_tuning;

/* Engine lifetime. ce_create selects `device` and allocates the engine's small
 * device scratch (work-queue cursor). */
int ce_create(ce_engine** out, int device);
void ce_destroy(ce_engine* e);
const char* ce_last_error(const ce_engine* e);
const char* ce_version(void);

/* Fixed molecule for ce_run / ce_run_device: n in 1..10 atoms, masses (electron
 * masses, > 0) and charges; pair constants k q_i q_j are formed in double and
 * narrowed to float like batched_integrator.hpp:79-87. */
int ce_set_molecule(ce_engine* e, int n, const double* mass_me, const double* charge,
                    double coulomb_k);
int ce_set_tuning(ce_engine* e, const ce_tuning* t);
/* The launch shape a plain-FP32 run of the current molecule uses (explicit
 * fields, else the autotuned entry, else the defaults: one thread per sim up to
 * 6 atoms (4 to 6 with Kahan compensation), two threads per sim from 7 atoms
 * (8 and 10 with Kahan compensation), else one lane per atom). */
int ce_get_tuning(const ce_engine* e, ce_tuning* t);

/* Integrate S explosions of the fixed molecule from rest.
 * pos: [S][N][3] float initial positions (host for ce_run, device for
 * ce_run_device). ce_run copies in, runs and copies out synchronously. In the
 * one-thread and two-thread layouts (2^15 <= S < 2^31, device buffers up to
 * 8 GiB) it is ONE launch over the whole batch with its copies streamed around
 * it: positions go up in up to 32 chunks that the kernel's warps wait for
 * (bounded), and each chunk's results come down as soon as the kernel has
 * finished its last sim (mapped-memory flags the host polls, bounded). Otherwise
 * it runs up to sixteen chunks (smaller at both ends) whose copies overlap the
 * integration of the neighbouring chunks (neighbouring chunks integrate on two
 * streams, so one chunk's last simulations overlap the next chunk's first).
 * Pinned host buffers let the copies overlap the integration;
 * ce_run_device enqueues on `stream` (cudaStream_t, NULL = legacy default) and
 * returns without synchronizing. S == 0 is a no-op. */
int ce_run(ce_engine* e, uint64_t S, const float* pos, const ce_run_config* cfg,
           const ce_outputs* out);
int ce_run_device(ce_engine* e, uint64_t S, const float* pos, const ce_run_config* cfg,
                  const ce_outputs* out, void* stream);

/* The Velocity Verlet strategy (IntegratorKind::VelocityVerlet,
 * src/integrators.cpp:14-47) under the same convergence driver
 * (src/driver.cpp:7-46) for the engine's molecule: fixed step dt =
 * cfg->max_dt, stop at PE <= pe_stop_fraction * PE_0 or max_steps, then the
 * energy rescale. IEEE FP32 in the reference's operation order, so results equal
 * the reference's scalar f32 engine bit for bit. rtol / atol are unused and
 * precision_mode must be 0. Device pointers, async on stream; outputs as
 * ce_run_device (rejects, positions and e0 are not written). */
int ce_run_verlet_device(ce_engine* e, uint64_t S, const float* pos, const ce_run_config* cfg,
                         const ce_outputs* out, void* stream);

/* Number of kernel launches the last ce_run / ce_run_device issued. */
int ce_last_launch_count(const ce_engine* e);

/* ---- mixed molecules ---------------------------------------------------
 * The reference builds one BatchedRK45 per molecule (all lanes share it,
 * include/coulomb/batched_force.hpp:8-13) and its scalar driver takes any
 * Molecule (src/driver.cpp:7); a mixed population therefore takes one reference
 * call per molecule. These entry points integrate any mix of 1..10-atom
 * molecules in one call. Rows are padded to CE_MAX_ATOMS atoms:
 *   n_atoms [S] uint8, mass_me [S][10] double, charge [S][10] double,
 *   pos [S][10][3] float;  out->momenta [S][10][3] float (rows past n untouched
 *   except for one-atom and invalid sims, which are zero-filled).
 * A sim with n outside 1..10 gets status CE_SIM_BAD_INPUT. S < 2^32. */
typedef struct ce_mixed_batch {
  const uint8_t* n_atoms;
  const double* mass_me;
  const double* charge;
  const float* pos;
} ce_mixed_batch;

#define CE_SCHEDULE_ONE_LAUNCH 0 /* one persistent launch walks the size buckets 10 -> 2 */
#define CE_SCHEDULE_PER_SIZE 1   /* one launch per size bucket, in sequence            */
#define CE_SCHEDULE_OVERLAP 2    /* the per-size launches alternating between the call's *
                                  * stream and an engine side stream, so each bucket's   *
                                  * last simulations overlap the next bucket's start;    *
                                  * results equal the other schedules' bit for bit       */

/* Size the engine's mixed-batch scratch (bucket tables + a 4-byte-per-sim
 * permutation) for up to S sims, so later calls, and graph captures, allocate
 * nothing. ce_run_mixed_device grows it on demand outside a capture. */
int ce_reserve_mixed(ce_engine* e, uint64_t S);
int ce_run_mixed_device(ce_engine* e, uint64_t S, const ce_mixed_batch* in, double coulomb_k,
                        const ce_run_config* cfg, const ce_outputs* out, int schedule, void* stream);
/* Integrator state of each sim, mixed layout (device pointers). No counterpart
 * in the reference, whose integrators keep this state in the object between
 * steps (src/integrators.cpp:63-147). A run given `save` writes, for every sim
 * it finishes, the state it stopped in: positions, velocities v (not m v), the
 * next step size h (0 unless the sim finished CE_SIM_OK), time, accepted steps,
 * rejected attempts, E0, and in the Kahan modes the compensation terms. A run
 * given `resume` (same precision mode and tolerances, a smaller pe_stop_fraction)
 * continues every sim whose saved h > 0 from that state, bit for bit as one
 * uninterrupted run would have; sims with h = 0 start from rest at in->pos. Its
 * steps / rejects / t outputs count from the start of the first run. Every
 * pointer is required, `comp` only in the Kahan modes. */
typedef struct ce_sim_state {
  float* positions;  /* [S][10][3] */
  float* velocities; /* [S][10][3] */
  float* h;          /* [S] */
  double* t;         /* [S] */
  uint32_t* steps;   /* [S] */
  uint32_t* rejects; /* [S] */
  double* e0;        /* [S] */
  float* comp;       /* [S][10][6]: x then v compensation (CE_PREC_KAHAN) */
} ce_sim_state;
/* ce_run_mixed_device with state: `resume` and `save` may each be NULL (and may
 * not share buffers). With either, the per-size schedule runs whatever
 * `schedule` says. */
int ce_run_mixed_device_state(ce_engine* e, uint64_t S, const ce_mixed_batch* in, double coulomb_k,
                              const ce_run_config* cfg, const ce_sim_state* resume, const ce_sim_state* save,
                              const ce_outputs* out, int schedule, void* stream);
/* Host buffers, synchronous; one-launch schedule unless ce_autotune_mixed found
 * the per-size schedule faster. Up to 8 chunks whose copies overlap the
 * neighbouring chunks' integration when the host buffers are pinned. Whole rows
 * come back: entries past n in out->momenta and out->positions are zero. */
int ce_run_mixed(ce_engine* e, uint64_t S, const ce_mixed_batch* in, double coulomb_k,
                 const ce_run_config* cfg, const ce_outputs* out);

/* ---- CUDA graphs ---------------------------------------------------------
 * Capture the engine calls issued on `stream` (non-default) between begin and
 * end into an instantiated graph; ce_graph_launch replays it on any stream.
 * The captured calls must not need to grow engine scratch (ce_reserve_mixed). */
typedef struct ce_graph ce_graph;
int ce_graph_begin(ce_engine* e, void* stream);
int ce_graph_end(ce_engine* e, void* stream, ce_graph** out);
int ce_graph_launch(ce_graph* g, void* stream);
void ce_graph_destroy(ce_graph* g);

/* ---- autotuner -----------------------------------------------------------
 * Time candidate launch shapes on the device -- threads per block (sims per
 * block), refill granularity, and the layout (fixed path: one thread per sim,
 * two threads per sim or one lane per atom; mixed path: one lane per atom or
 * two threads per sim) -- over the caller's device inputs, and keep the
 * fastest in the engine; it then applies wherever the matching ce_tuning field
 * is 0 (fixed path: per atom count; mixed path: one entry, plus the faster
 * schedule in *best_schedule). `report` (may be NULL) receives up to `cap`
 * candidates with their measured sims/s; *n_report their number. */
typedef struct ce_tune_result {
  ce_tuning t;
  double sims_per_s;
  int32_t schedule;
} ce_tune_result;
int ce_autotune_fixed(ce_engine* e, uint64_t S, const float* pos_dev, const ce_run_config* cfg,
                      ce_tune_result* report, int cap, int* n_report);
int ce_autotune_mixed(ce_engine* e, uint64_t S, const ce_mixed_batch* dev_in, double coulomb_k,
                      const ce_run_config* cfg, ce_tune_result* report, int cap, int* n_report,
                      int* best_schedule);

/* ce_run_device for callers that cannot allocate device memory. No counterpart
 * in the reference. It needs no engine: the molecule comes with the call, the
 * inputs and outputs are the caller's device buffers (as for ce_run_device), and
 * the kernel's only scratch, its work-queue cursor, lives in a 256-byte static
 * device array that every GPU loading this library holds until exit. Nothing
 * here calls cudaMalloc, cudaFree or an allocating library routine.
 * Limits: 1 <= n <= 10 atoms and S <= 2^40 sims; anything outside is rejected
 * with CE_ERR_INVALID before a launch. The first call on a device (that device
 * current) resolves the array's address once, so make it before any stream
 * capture. The address is kept for the life of the process: a cudaDeviceReset
 * (or any teardown of the device's primary context) between calls is not
 * supported, as the array may then move. All calls share the cursor: each call clears it on `stream` first, and
 * calls that overlap on the GPU race on it. `err` (may be NULL) receives a
 * message of at most err_len bytes on failure. */
int ce_run_device_noalloc(int n, const double* mass_me, const double* charge, double coulomb_k,
                          uint64_t S, const float* pos, const ce_run_config* cfg,
                          const ce_outputs* out, void* stream, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif /* CE_GPU_H */
