/* sinksim-b200: the C ABI of the B200 batch flooding engine (libsinksim_b200.so).
 *
 * A drop-in for the batch path of the reference sinksim engine: the same compiled ship / sim / sweep files, the
 * same per-instance connection setters and the same batch-results, curves, events and traces. Each entry point
 * names the reference interface it replaces (paths are files of the reference repository).
 *
 * Conventions: plain pointers and sizes only. Every function returns SSB_OK (0) on success or a negative SSB_E*
 * code; ssb_last_error() then describes the failure (thread-local, valid until the next call on that thread).
 * Handles are not thread-safe; use one per thread. Numerics: 0 = "portable" (double precision), 1 = "portable32"
 * (single-precision column partials); the reference's "oracle" and "std" numerics exist on its CPU only and are
 * rejected here (SSB_EUNSUPPORTED), as the reference's GPU runner rejects them (apps/sinksim_cuda_run.cpp:171-175).
 *
 * State records use the reference trace record layout (engine/src/trace.cpp:140-150): t, zO, pitch, roll, vz,
 * wth, wph, inflow, Vb, hullTop, then vol, level, cx, cy, cz for each of the N nodes: 10 + 5 N doubles.
 * Readout records are 7 doubles: t, trim (deg), list (deg), water (t), inflow (t/min), draftF, draftA
 * (engine/include/sinksim/cuda/batch.hpp:39-43).
 */
#ifndef SINKSIM_B200_H
#define SINKSIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SSB_OK 0
#define SSB_EINVAL (-1)       /* bad argument: the reference throws std::invalid_argument / std::out_of_range */
#define SSB_ERUNTIME (-2)     /* I/O, format, hash or CUDA failure: the reference throws std::runtime_error */
#define SSB_ESTATE (-3)       /* call out of order (set after run, result before run): std::logic_error */
#define SSB_EUNSUPPORTED (-4) /* a numerics or option the GPU engine does not provide */
#define SSB_ENODEVICE (-5)    /* no usable CUDA device */

typedef struct ssb_batch ssb_batch;

/* Options of a batch: engine/include/sinksim/cuda/batch.hpp:27-37 (BatchOptions), plus the launch shape and the
 * batching workloads' extra retire rule. Initialise with ssb_batch_options_init. */
typedef struct ssb_batch_options {
  int32_t count;             /* instances (>= 1) */
  int32_t numerics;          /* 0 portable, 1 portable32 (the reference's mixedPrecision) */
  int32_t traced_instances;  /* leading instances that record traces */
  int32_t dense_steps;       /* dense records at the start of each trace */
  double sample_every;       /* s between sampled trace records */
  double curve_every;        /* s between readout-curve records of every instance; 0: none */
  double t_max;              /* s: every instance stops here if it has not foundered */
  int64_t steps_per_launch;  /* 0: one persistent launch; > 0: bounded launches (the reference's stepsPerLaunch) */
  int32_t team_warps;        /* warps stepping one simulation in the main phase: 1, 2, 4, 8 or 16; 0: chosen */
  int32_t tail_team_warps;   /* warps per simulation of the last phase (the phases double the team size up to it): 8 or
                                16 (a whole 512-thread block per simulation); 0 no tail phase, -1 chosen */
  int32_t teams_per_block;   /* simulations per block in the main phase; 0: chosen */
  int32_t yield_below;       /* the main phase hands its instances to the tail phase once at most this many remain;
                                -1: from handover_factor */
  int32_t blocks;            /* main-phase grid size; 0: persistent grid sized to the device */
  int32_t device;            /* CUDA device ordinal */
  /* extra retire rule (disabled when rule_enabled == 0): an instance stops once |pitch| > rule_pitch and the deck
   * edge point (rule_x, +-rule_y, rule_z) is below the sea ("sink"), or once |pitch rate| < rule_wth has held for
   * rule_settle seconds ("settle"). It never changes the physics. */
  int32_t rule_enabled;
  double rule_pitch, rule_x, rule_y, rule_z, rule_wth, rule_settle;
  /* the reference's calm rule of Simulation::run (engine/src/simulation.cpp:179-182), a sweep's "stopWhenStable":
   * after 1,800 s an instance stops once |inflow| < 0.02, |pitch rate| < 1e-5 and |heave rate| < 1e-3 have held for
   * more than 1,200 s (stop reason 5). Exclusive with the retire rule. */
  int32_t stop_when_stable;
  /* a launch phase hands its unfinished instances to the next (twice the warps per simulation) once they number at
   * most this multiple of the next phase's resident simulations; 0: the default (2) */
  double handover_factor;
  /* the claim order of the launch phases after the first: 0 (the default) the unfinished instances with the fewest
   * steps done first, so that the runs with the most work left get the larger teams first; 1 by index. The results
   * are the same either way. */
  int32_t claim_by_index;
  /* 1: every block first copies the model's column table (the arrays the buoyancy integral reads, 40 bytes a column
   * in portable numerics, 20 in portable32) into its shared memory beside its simulations' slots, by bulk
   * asynchronous copies, and the buoyancy reads it from there; a phase whose blocks lack the room runs fewer
   * simulations per block. Single-model batches only; the results are the same either way. 0 (the default): the
   * table is read from global memory through the L1 cache. */
  int32_t stage_columns;
} ssb_batch_options;

typedef struct ssb_device_info {
  char name[256];
  int32_t major, minor, multiprocessors;
  uint64_t global_memory, shared_per_block_optin;
  int32_t runtime_version, driver_version;
} ssb_device_info;

/* Summary of one instance after a run: engine/include/sinksim/cuda/batch.hpp:45-54 (InstanceResult). */
typedef struct ssb_instance_summary {
  int32_t foundered;
  int32_t stop_reason; /* 1 foundered, 2 tMax, 3 sink rule, 4 settle rule, 5 stable (calm rule), 0 still running */
  double founder_t, t_end;
  int64_t steps;
  int32_t event_count;
  int32_t curve_count;  /* records of ssb_batch_curve, the final record included */
  double outputs[7];    /* inflow, Vb, hullTop, mw, bx, by, bz of the last step */
} ssb_instance_summary;

/* The launch shape the engine chose: the main phase and the tail phase (tail_team_warps == 0: none). */
typedef struct ssb_launch_info {
  int32_t team_warps, teams_per_block, blocks, blocks_per_sm, yield_below;
  int32_t tail_team_warps, tail_teams_per_block, tail_blocks, tail_blocks_per_sm;
  uint64_t slot_bytes;  /* shared memory of one simulation */
  int32_t phases;       /* launch phases of one run: from the main team size up to the tail's */
  int32_t kernels;      /* kernel launches of one run to the end: the counters' reset, the phases and, before each
                           phase after the first, the two kernels of its claim order */
  int32_t staged_phases; /* phases whose blocks hold the column table in shared memory (stage_columns) */
} ssb_launch_info;

/* The message of the last failure on this thread. */
const char* ssb_last_error(void);
/* Library version string. */
const char* ssb_version(void);

/* Is a CUDA device present? Returns 1 or 0; `why` (may be NULL) receives the reason. cuda::available,
 * engine/include/sinksim/cuda/batch.hpp:17. */
int ssb_available(char* why, size_t why_cap);
/* cuda::device_info, engine/include/sinksim/cuda/batch.hpp:19-25. */
int ssb_get_device_info(int32_t device, ssb_device_info* out);

void ssb_batch_options_init(ssb_batch_options* opt);

/* Loads and verifies a compiled ship and sim (io::load_ship / io::load_sim / io::check_pairing,
 * engine/src/compiled.cpp:108-279) and creates a batch of opt->count instances of it
 * (cuda::Batch::Batch, engine/cuda/batch.cu:170-209). */
int ssb_batch_create(const char* ship_path, const char* sim_path, const ssb_batch_options* opt, ssb_batch** out);
/* A fleet: instances of several compiled models in one batch, stepped in the same launches (no counterpart in the
 * reference, which runs one model per batch). instance_model[i] (opt->count entries) picks instance i's model among
 * the n_models ship/sim pairs. Per-instance setters, runs, summaries, states, events, curves and final readouts work
 * as for one model, with each instance's own node and connection counts (ssb_batch_instance_shape); sweeps, traces,
 * batch-results files and the no-allocation run take a batch of one model and return SSB_EINVAL / SSB_ESTATE here. */
int ssb_fleet_create(int32_t n_models, const char* const* ship_paths, const char* const* sim_paths, const int32_t* instance_model,
                     const ssb_batch_options* opt, ssb_batch** out);
/* Instance i's model (index into the fleet's models; 0 for a batch of one model), node count and connection count. */
int ssb_batch_instance_shape(const ssb_batch* b, int32_t instance, int32_t* model, int32_t* nodes, int32_t* connections);
void ssb_batch_destroy(ssb_batch* b);
int ssb_batch_nodes(const ssb_batch* b, int32_t* nodes, int32_t* connections);
int ssb_batch_launch_info(const ssb_batch* b, ssb_launch_info* out);
/* The kernel launches that one run to the end captures into its CUDA graph, in order, for a batch with these options
 * and phases whose hand-over bounds are yield_below[0 .. n_phases-1] (phase k pauses once at most yield_below[k]
 * instances remain; the last phase's is 0). kinds[i] is 0 for the counters' reset, 1 for the claim-order pair of
 * kernels (list and rank the unfinished instances) and 2 for a phase's batch kernel; phases[i] is the phase it belongs
 * to (-1 for the reset). *n receives the step count; at most cap steps are written (SSB_EINVAL if cap is too small).
 * Host-only: needs no device. No counterpart in the reference, which launches in host-driven chunks. */
int ssb_launch_plan(const ssb_batch_options* opt, int32_t n_phases, const int32_t* yield_below, int32_t* kinds, int32_t* phases,
                    int32_t cap, int32_t* n);

/* Per-instance setup before the run: cuda::Batch::restore / set_connection_enabled / set_connection_area /
 * set_connection_activation (engine/cuda/batch.cu:217-243). */
int ssb_batch_restore(ssb_batch* b, int32_t instance, const double* record);
int ssb_batch_set_connection_enabled(ssb_batch* b, int32_t instance, int32_t connection, int32_t enabled);
int ssb_batch_set_connection_area(ssb_batch* b, int32_t instance, int32_t connection, double area);
int ssb_batch_set_connection_activation(ssb_batch* b, int32_t instance, int32_t connection, double t_on);
/* ssb_batch_set_connection_area over a block of instances: the area of connection connections[j] of instance first + i
 * is areas[i * n_connections + j] (row-major, count x n_connections). Every index is checked before anything is
 * written: on an error (SSB_EINVAL, or SSB_ESTATE after the run) nothing changes. No counterpart in the
 * reference, whose setters take one value per call; one call here replaces count x n_connections of them. */
int ssb_batch_set_connection_areas(ssb_batch* b, int32_t first, int32_t count, int32_t n_connections, const int32_t* connections,
                                   const double* areas);
/* The order in which the first launch phase claims the instances: order[0 .. n) a permutation of 0 .. count-1
 * (n == count; SSB_EINVAL otherwise, SSB_ESTATE after the run). A caller who knows which runs are long (an earlier
 * evaluation of similar points) lists them first, so that they do not start last and end the batch late; the
 * default is by index. The results do not depend on it. No counterpart in the reference, which launches every
 * instance of a chunk at once. */
int ssb_batch_set_claim_order(ssb_batch* b, const int32_t* order, int32_t n);
/* Instance i takes instance i of a sweep file: sweep::apply (engine/include/sinksim/sweep.hpp:49-65) through the
 * setters above, as sinksim_cuda_run --sweep does (apps/sinksim_cuda_run.cpp:37-41). The sweep must have exactly
 * opt->count instances. */
int ssb_batch_apply_sweep(ssb_batch* b, const char* sweep_path);
/* Instance i takes instance first + i of a sweep file: one GPU's contiguous shard of a sweep run on several GPUs.
 * Saved results name the instances by those sweep instances' ids. No counterpart in the reference, which runs a
 * sweep on one GPU; the per-instance setup is sweep::apply as above. */
int ssb_batch_apply_sweep_range(ssb_batch* b, const char* sweep_path, int32_t first);

/* cuda::Batch::run (engine/cuda/batch.cu:245-308): uploads the instances, runs every one to its end, downloads the
 * results. *seconds (may be NULL) receives the wall time. */
int ssb_batch_run(ssb_batch* b, double* seconds);
/* The same in three parts, for callers that time the device alone: ssb_batch_launch's *device_ms is measured with
 * CUDA events on the engine's stream around the kernel launches. */
int ssb_batch_upload(ssb_batch* b);
/* Makes a finished batch runnable again from its staged inputs (initial states and connection fields as set):
 * repeated runs of one batch, for calibration loops and benchmarks. No counterpart in the reference, whose
 * cuda::Batch::run throws when called twice (engine/cuda/batch.cu:246). */
int ssb_batch_reset(ssb_batch* b);
int ssb_batch_launch(ssb_batch* b, float* device_ms);
int ssb_batch_download(ssb_batch* b);
/* Bytes one run copies host to device and device to host (inputs and results). */
int ssb_batch_transfer_bytes(const ssb_batch* b, uint64_t* h2d, uint64_t* d2h);
/* The last launch by phase (0 .. ssb_launch_info.phases - 1): the phase's team size, its device time in milliseconds
 * (CUDA events around its kernel launches) and the steps its kernels took. No counterpart in the reference, whose run
 * is one phase; it serves the per-kernel roofline of the benchmark. */
int ssb_batch_phase_stats(const ssb_batch* b, int32_t phase, int32_t* team_warps, float* device_ms, int64_t* steps);

/* Results after the run: cuda::Batch::total_steps / result / curve / final_readouts / trace
 * (engine/cuda/batch.cu:302-400). */
int ssb_batch_total_steps(const ssb_batch* b, int64_t* steps);
int ssb_batch_summary(const ssb_batch* b, int32_t instance, ssb_instance_summary* out);
int ssb_batch_state(const ssb_batch* b, int32_t instance, double* record);
/* Events in firing order: time, index (monitor or mark; -1 for the founder) and kind (0 overflow, 1 mark,
 * 2 founder). Writes at most cap; returns the count through *count. */
int ssb_batch_events(const ssb_batch* b, int32_t instance, double* t, int32_t* id, int32_t* kind, int32_t cap, int32_t* count);
/* The readout curve (7 values per record), closed by the final readouts; at most cap records. */
int ssb_batch_curve(const ssb_batch* b, int32_t instance, double* records, int32_t cap, int32_t* count);
int ssb_batch_final_readouts(const ssb_batch* b, int32_t instance, double* record7);
/* io::save_trace of cuda::Batch::trace(instance) (engine/src/trace.cpp:272-308). */
int ssb_batch_save_trace(const ssb_batch* b, int32_t instance, const char* path);
/* sweep::save_results of the batch (engine/src/sweep.cpp:163-201); instance ids come from the sweep file when
 * sweep_path is not NULL. */
int ssb_batch_save_results(const ssb_batch* b, const char* sweep_path, const char* results_path);

/* sinksim_cuda_run --sweep (apps/sinksim_cuda_run.cpp:26-83) in one call: numerics "portable" or "portable32".
 * *steps and *seconds (may be NULL) receive the aggregate steps and the wall time. */
int ssb_run_sweep(const char* ship_path, const char* sim_path, const char* sweep_path, const char* numerics, const char* results_path,
                  int64_t* steps, double* seconds);
/* ssb_run_sweep on instances [first, first + count) of the sweep (count < 0: to its end) on CUDA device `device`:
 * one GPU's shard of a sweep run on several GPUs (one process per GPU). The results name the instances by their
 * sweep ids. No counterpart in the reference, whose GPU runner takes a whole sweep on one GPU. */
int ssb_run_sweep_range(const char* ship_path, const char* sim_path, const char* sweep_path, const char* numerics, int32_t first,
                        int32_t count, int32_t device, const char* results_path, int64_t* steps, double* seconds);
/* sinksim_sweep --compare (apps/sinksim_sweep.cpp:19-31, engine/src/sweep.cpp:234-281): exact comparison.
 * *differing receives the count of differing values; first (may be NULL) the first difference. */
int ssb_compare_results(const char* a_path, const char* b_path, uint64_t* compared, uint64_t* differing, char* first, size_t first_cap);

/* The portable math of the engine, evaluated on the host and on the device (for parity checks of the device
 * code): op 0 sin(x), 1 cos(x), 2 pow(x, y), 3 scalbn(x, (int)y). The reference's fdlibm port,
 * engine/include/sinksim/kernel/fdlibm_portable.hpp:71-435. */
int ssb_portable_math_host(int32_t op, const double* x, const double* y, double* out, int64_t n);
int ssb_portable_math_device(int32_t op, const double* x, const double* y, double* out, int64_t n);

/* Runs `count` instances of the batch's model without allocating any device memory, for callers that cannot call
 * cudaMalloc at run time: a host application that owns every device allocation through its own memory pool (a
 * calibration or control loop embedded in a larger program), or code that must not allocate once it is running.
 * No counterpart in the reference, whose cuda::Batch allocates everything itself (engine/cuda/batch.cu:23-59).
 *
 * All pointers are the caller's device memory: state (count x 8 doubles: t, zO, pitch, roll, vz, wth, wph, then a
 * 0 for the settle timer of the retire rule), vol, level, cx, cy, cz (count x N each) are read as the initial states
 * and overwritten with the final ones; en (bytes), area, t_on (count x connections each) are the connection fields;
 * final_readouts (count x 7) receives each instance's final readouts, steps (int64) its step count and stop_reason its
 * stop (1 foundered, 2 t_max, 3 sink rule, 4 settle rule, 5 stable under the calm rule). Numerics, t_max, the retire
 * rule and the calm rule (stop_when_stable) are the batch's options; curves and traces are not recorded. `stream` is a
 * cudaStream_t (NULL: the default stream); the call returns once the work is queued on it.
 *
 * The kernel's scratch (the work-queue head, the count of unfinished instances, each instance's outputs, event log,
 * overflow and mark times) lives in a fixed 4 MiB device array of the library, which every GPU that loads the library
 * holds until the process exits; a count whose scratch does not fit returns SSB_EINVAL with the largest count that
 * would. The first call on a device sets up that array's device address (cudaGetSymbolAddress with the device
 * current), so make it before any stream capture; later calls query the address again (no allocation). Every call also
 * makes host-side runtime calls that allocate nothing (cudaSetDevice, cudaFuncSetAttribute for the team size it picks,
 * an occupancy query). Every call shares the array and clears what must start at zero; calls that overlap on the GPU
 * race on it. The batch handle must have been created beforehand (which allocates). */
int ssb_batch_run_noalloc(const ssb_batch* b, int32_t count, const uint8_t* en, const double* area, const double* t_on, double* state,
                          double* vol, double* level, double* cx, double* cy, double* cz, double* final_readouts, int64_t* steps,
                          int32_t* stop_reason, void* stream);

/* ------------------------------------------------------------------------------------------------ the adjoint
 * Gradients of a trajectory objective with respect to every connection area, for many instances of one compiled
 * model, by a hand-written discrete adjoint of the portable (FP64) time step with checkpoints every K steps and
 * recomputation in between. No counterpart in the reference, which has no gradients
 * (docs/adr/0001-single-source-cpp-kernel.md:25-26); instances are set up like cuda::Batch's
 * (engine/cuda/batch.cu:217-243).
 *
 * Each instance runs from the compiled initial state until t_max or its founder. The objective of instance i is
 * J_i = sum_k (trim(s_k) - trim_i,k)^2 + (heave(s_k) - heave_i,k)^2 with trim in degrees (kernel/readouts.hpp:27) and
 * heave the mean of the forward and aft drafts (:31-32), at the states s_k where a readout curve recorded every sample
 * time would take its records (the first step start with t >= times[k]; the final state once the run has stopped).
 * The gradient is d J_i / d area[c] along the branch path the run takes. */
typedef struct ssb_adjoint ssb_adjoint;

/* count instances; checkpoint_every steps between checkpoints (256 if 0); team_warps 4, 8 or 16 (0: 16 for at most two
 * instances per SM, else 8). */
int ssb_adjoint_create(const char* ship_path, const char* sim_path, int32_t count, double t_max, int32_t checkpoint_every,
                       int32_t team_warps, int32_t device, ssb_adjoint** out);
void ssb_adjoint_destroy(ssb_adjoint* a);
int ssb_adjoint_set_connection_enabled(ssb_adjoint* a, int32_t instance, int32_t connection, int32_t enabled);
/* As ssb_batch_set_connection_areas: areas[i * n_connections + j] for connection connections[j] of instance first + i. */
int ssb_adjoint_set_connection_areas(ssb_adjoint* a, int32_t first, int32_t count, int32_t n_connections, const int32_t* connections,
                                     const double* areas);
/* n sample times (ascending) and the targets trim[i * n + k], heave[i * n + k] of every instance. */
int ssb_adjoint_set_objective(ssb_adjoint* a, int32_t n, const double* times, const double* trim, const double* heave);
/* The order in which the adjoint's teams claim the instances: order[0 .. n) a permutation of 0 .. count-1 (n == count;
 * SSB_EINVAL otherwise), or order NULL / n 0 for index order (the default). When there are more instances than teams,
 * the longest runs listed first (known from an earlier evaluation of similar points) end the call sooner. The results
 * do not depend on it. */
int ssb_adjoint_set_claim_order(ssb_adjoint* a, const int32_t* order, int32_t n);
/* Memory for step records, all teams together, in bytes. A team keeps the records of its run's last steps in a ring
 * of budget / teams bytes, at least one segment (checkpoint_every records of the largest size); the reverse recomputes
 * from its checkpoint only a segment the ring no longer holds. 0, the default: room for a whole run of t_max with two
 * level passes per node (about 15 KB a step on a 64-space model), within half the device memory free at the next run.
 * The results do not depend on it. */
int ssb_adjoint_set_tape_budget(ssb_adjoint* a, uint64_t bytes);
/* The ring of each team in the last run, in bytes. */
int ssb_adjoint_ring_bytes(const ssb_adjoint* a, uint64_t* bytes);
/* Runs every instance forward and back. J (count), grad (count x connections, row-major), steps (count) and error
 * (count; nonzero where a step took a branch without an adjoint) may be NULL; device_ms receives the kernel's time. */
int ssb_adjoint_run(ssb_adjoint* a, double* J, double* grad, int64_t* steps, int32_t* error, float* device_ms);
/* The run's trim and heave at the sample times (count x n each). */
int ssb_adjoint_samples(const ssb_adjoint* a, double* trim, double* heave);
/* Connections, team size and teams of the last run; bytes sent to and read back from the device in the last run. */
int ssb_adjoint_info(const ssb_adjoint* a, int32_t* connections, int32_t* team_warps, int32_t* teams, uint64_t* h2d_bytes, uint64_t* d2h_bytes);
/* Where the last run's time went, per instance (count x 3, row-major, nanoseconds of the device's global timer while
 * the instance's team worked on it): the forward run with its checkpoints, the recomputation of segments from their
 * checkpoints, the reverse steps. */
int ssb_adjoint_phase_times(const ssb_adjoint* a, int64_t* ns);
/* Steps each instance recomputed from its checkpoints in the last run (count): 0 when its ring held the whole run. */
int ssb_adjoint_recomputed_steps(const ssb_adjoint* a, int64_t* steps);

/* Measured rate of separately rounded adds and multiplies on the device (fp64 = 1: double, 0: float), the
 * denominator of the engine's roofline; operations per second through *ops_per_s. No counterpart in the reference. */
int ssb_measure_add_mul_peak(int32_t fp64, int32_t device, double* ops_per_s);

/* Health of the last run: *flags receives 0, or bit 1 when an instance's rigid-body state (heave, pitch, roll or a rate)
 * was not finite when the kernel stored it (a NaN or infinity in an input, or a diverging model). The reference has no
 * such report; its engine computes on with NaNs. The results are unchanged; this says that some cannot be trusted.
 * Bit 2: with stage_columns, a block's copy of the column table did not arrive within its wait limit and that block
 * read the table from global memory (the results are the same). */
int ssb_batch_health(const ssb_batch* b, int32_t* flags);

/* Loads and verifies a compiled ship and sim without running anything (no device needed): formats and versions,
 * every array's length and integer range, every array's FNV-1a hash and the chained hash against the ones the files
 * state, and that the sim was compiled for this ship (io::load_ship / io::load_sim / io::check_pairing,
 * engine/src/compiled.cpp:82-279). SSB_ERUNTIME with the first problem found (ssb_last_error), else SSB_OK. */
int ssb_check_model(const char* ship_path, const char* sim_path);
/* The same checks, then a sweep file against that sim (sweep::load_sweep, engine/src/sweep.cpp:25-70): its format,
 * version and the connection kinds it names. */
int ssb_check_sweep(const char* ship_path, const char* sim_path, const char* sweep_path);

/* FNV-1a 64-bit over n bytes, continuing from `state` (0xcbf29ce484222325 to start): the hash the compiled-file
 * loaders verify (the reference's engine/include/sinksim/hash.hpp and tools/js/lib/fnv.js), for writers of compiled
 * files such as the hull compiler. Needs no device. */
uint64_t ssb_fnv1a64(uint64_t state, const void* data, size_t n);

#ifdef __cplusplus
}
#endif

#endif
