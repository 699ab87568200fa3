/*
 * spinsim_b200 C ABI: the B200 (sm_100a) evaluation path of spinsim behind plain C entry points.
 *
 * The reference (alexander-tritt-monash/spinsim) is one Python module on numba; its evaluation path
 * is Simulator(...).evaluate(...) -> Results(time, time_evolution, state, spin).  Each entry point
 * below names the reference function it replaces (spinsim/__init__.py:line).
 *
 * Conventions
 *  - Every function returns 0 (SPINSIM_OK) or a negative SPINSIM_ERR_* code; the message of the most
 *    recent failure on the calling thread is available from spinsim_last_error().
 *  - Array arguments named *_dev are device pointers (any allocator).  Complex arrays are interleaved
 *    (re, im) doubles, numpy complex128 layout.  Output layouts match the reference's numpy outputs:
 *      time[N] f64, time_evolution U[N][d][d] c128, state[N][d] c128, spin[N][3] f64.
 *  - `stream` is a cudaStream_t (NULL = legacy default stream).  All work is stream-ordered.  The
 *    single-instance entry points (spinsim_evaluate, spinsim_time_evolution, spinsim_state,
 *    spinsim_state_static, spinsim_piece_*) and spinsim_batch_launch only launch kernels: their
 *    descriptors travel as launch arguments and are written into the workspace on the device, so
 *    they never wait for the stream and can be captured into a CUDA graph (host arrays such as psi0
 *    are read during the call).  Host waits: spinsim_plan_create (module load; with a user field,
 *    the link), spinsim_batch_prepare (copies from pageable host memory, which wait for the stream;
 *    spinsim_batch_prepare_staged copies from the caller's page-locked staging instead), and the
 *    first spinsim_state_static call on a device (it looks up the library's scratch array).
 *  - The library allocates no device memory on the evaluation path.  Scratch comes from the caller's
 *    workspace, sized by the *_workspace_size queries (256-byte aligned start required).
 */
#ifndef SPINSIM_B200_H
#define SPINSIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPINSIM_OK 0
#define SPINSIM_ERR_INVALID (-1)     /* bad argument (message says which) */
#define SPINSIM_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define SPINSIM_ERR_LINK (-3)        /* nvJitLink / module load of a user field failed */
#define SPINSIM_ERR_UNSUPPORTED (-4) /* method combination not built */
#define SPINSIM_ERR_WORKSPACE (-5)   /* workspace too small or misaligned */

/* Method enumerations: the values of the reference's IntegrationMethod (I:68-93) order and
 * ExponentiationMethod.index (I:95-129). */
#define SPINSIM_INTEGRATION_MAGNUS_CF4 0
#define SPINSIM_INTEGRATION_EULER 1
#define SPINSIM_INTEGRATION_HEUN 2
#define SPINSIM_EXPONENTIATION_ANALYTIC 0
#define SPINSIM_EXPONENTIATION_LIE_TROTTER 1
#define SPINSIM_EXPONENTIATION_LIE_TROTTER_8 2
#define SPINSIM_FIELD_USER 0  /* user get_field linked from LTO-IR (field_ltoir in plan_create) */
#define SPINSIM_FIELD_TABLE 1 /* per-channel interpolation tables */
#define SPINSIM_FIELD_TONES 2 /* per-channel bias + sum of sinusoids */
#define SPINSIM_PRECISION_FP64 0
#define SPINSIM_PRECISION_FP32_BULK 1
/* Kernel of FP32-bulk plans with tone fields (spinsim_plan_desc.variant): the field samples of a
 * tile of output intervals as FP64 tensor-core matrix products (the default), or a warp-synchronous
 * phasor synthesis. */
#define SPINSIM_VARIANT_TENSOR 0
#define SPINSIM_VARIANT_SYNTH 1

/* Plan description: the compile-time specialisation of the reference's compile_time_evolver
 * (I:453-991), i.e. Simulator.__init__ (I:375) minus the user callable. */
typedef struct {
    int32_t spin_dim;          /* 2 (SpinQuantumNumber.HALF), 3 (ONE), or 0 for a mixed batch */
    int32_t integration;       /* SPINSIM_INTEGRATION_* */
    int32_t expo_half;         /* exponentiation for dimension-2 instances */
    int32_t expo_one;          /* exponentiation for dimension-3 instances */
    int32_t rotating;          /* use_rotating_frame */
    int32_t number_of_squares; /* number_of_squares (north_star: trotter_cutoff), >= 0 */
    int32_t field_kind;        /* SPINSIM_FIELD_* */
    int32_t precision;         /* SPINSIM_PRECISION_* */
    int32_t threads_per_block; /* 0 = library default (128); else a multiple of 32, <= 128 */
    int32_t max_registers;     /* 0 = no cap; <= 128 selects the 128-register build (built-in fields)
                                  or is passed to the JIT linker (user fields) */
    int32_t lanes;             /* lanes per output interval: 0 = auto, else 1, 2, 4, 8, 16 or 32 */
    int32_t variant;           /* SPINSIM_VARIANT_* (FP32-bulk tone plans; ignored otherwise) */
} spinsim_plan_desc;

/* One interpolation table: generate_interpolation_sampler's (time, amplitude, order,
 * zero_boundary) (I:1941-2147).  time/amplitude are device pointers; size 0 = no table. */
typedef struct {
    const double* time;
    const double* amplitude;
    int64_t size;
    int32_t order;
    int32_t zero_boundary;
} spinsim_table;

/* Per-instance field (host struct whose pointers are device pointers).  Channel c (x, y, z, q,
 * u1, u2, v1, v2) = bias[c] + gain[c] * source_c(t); source_c is tables[c] (FIELD_TABLE) or
 * sum_k A_k sin(w_k t + phi_k) over tones[3 * (tone_start[c] + k) ...] as (w, A, phi)
 * (FIELD_TONES).  FIELD_USER uses only params/n_params: the sweep_parameters of evaluate (I:993),
 * handed to the user's get_field. */
typedef struct {
    const double* params;
    int64_t n_params;
    const spinsim_table* tables; /* device array [8] */
    const double* tones;         /* device array */
    int32_t tone_start[8];
    int32_t tone_count[8];
    double bias[8];
    double gain[8];
} spinsim_field;

/* One evaluate() call inside a batch.  n_out and n_fine follow I:1025-1034 (use
 * spinsim_normalise_steps).  Offsets place the instance in the flat output arrays: out_offset in
 * intervals (time, spin), u_offset and state_offset in doubles. */
typedef struct {
    double t0;
    double dt_int;
    double dt_out;
    int64_t n_out;
    int64_t out_offset;
    int64_t u_offset;
    int64_t state_offset;
    int32_t n_fine;
    int32_t dim;
    int32_t field;  /* index into the batch's field array */
    int32_t interval0; /* time index of this instance's output step 0: time[i] = t0 + dt_out * (interval0 + i),
                        * as in I:818; 0 for a whole evaluate(), the first index of a piece when one
                        * evaluate() is split across launches or GPUs */
    double psi0[6]; /* complex[dim] interleaved */
} spinsim_instance;

typedef struct spinsim_plan spinsim_plan;
typedef struct spinsim_batch spinsim_batch;

typedef struct {
    int32_t registers_per_thread;
    int32_t threads_per_block;
    int32_t blocks_per_sm;  /* occupancy of the time-evolution kernel */
    int32_t sm_count;
    int32_t lanes;
    int32_t linked;         /* 1 if the kernel came from nvJitLink (user field) */
    int32_t variant;        /* SPINSIM_VARIANT_* in use for FP32-bulk tone plans, -1 for other plans */
    int32_t tile_intervals; /* output intervals per scheduling tile (a warp's, or a CTA's for the tensor path) */
} spinsim_plan_info;

/* Library version string. */
const char* spinsim_version(void);

/* Message of the last failure on this thread (copied into buf, NUL-terminated); returns its length. */
int spinsim_last_error(char* buf, size_t n);

/* Step normalisation of Simulator.evaluate, I:1025-1034: dt_int <- dt_out / round(max(dt_out/dt_int, 1)),
 * N = int((t1 - t0) / dt_out), K = floor(dt_out / dt_int + 0.5).  *warned is set when the reference
 * prints its non-integer-ratio warning (I:1027-1028). */
int spinsim_normalise_steps(double t0, double t1, double dt_int, double dt_out, double* dt_int_out, int64_t* n_out,
                            int32_t* n_fine, int32_t* warned);

/* Build a plan: replaces compile_time_evolver (I:453-991).  For SPINSIM_FIELD_USER, field_ltoir holds
 * the LTO-IR of `void spinsim_user_field(double t, double* sweep_parameters, int64_t n, double* field)`
 * (field[0..8) pre-zeroed by the caller), which is linked into the kernel with nvJitLink; otherwise
 * field_ltoir must be NULL.  Loads the module on the current device. */
int spinsim_plan_create(const spinsim_plan_desc* desc, const void* field_ltoir, size_t field_ltoir_size,
                        spinsim_plan** out);
int spinsim_plan_destroy(spinsim_plan* plan);
int spinsim_plan_get_info(const spinsim_plan* plan, spinsim_plan_info* info);

/* Simulator.evaluate for one instance (I:993-1085): time evolution (get_time_evolution, I:855-896),
 * state propagation (get_state, I:1089-1111, here a parallel scan) and, if spin_dev is non-NULL,
 * the spin expectation (get_spin, I:899-959).  field is a host struct; psi0 a host complex[d] array. */
size_t spinsim_evaluate_workspace_size(const spinsim_plan* plan, int64_t n_out);
int spinsim_evaluate(const spinsim_plan* plan, const spinsim_field* field, double t0, double dt_int, double dt_out,
                     int64_t n_out, const double* psi0, double* time_dev, double* u_dev, double* state_dev,
                     double* spin_dev, void* workspace_dev, size_t workspace_bytes, void* stream);

/* spinsim_evaluate plus, for an FP32-bulk plan, the scale of its rounding error: step_norms_dev[i]
 * receives, for output step i, the sum over its fine steps of |g|^2, g the step generators rounded
 * to FP32 (the reference has no FP32 form; its results carry no error statement).  The FP32 rounding
 * errors of the steps are independent, so the final state's error against the FP64 form is of order
 * 2^-24 sqrt(sum over all steps of |g|^2); spinsim_b200.Results.error_estimate states it.
 * step_norms_dev may be NULL; an FP64 plan does not write it. */
int spinsim_evaluate_with_norms(const spinsim_plan* plan, const spinsim_field* field, double t0, double dt_int,
                                double dt_out, int64_t n_out, const double* psi0, double* time_dev, double* u_dev,
                                double* state_dev, double* spin_dev, float* step_norms_dev, void* workspace_dev,
                                size_t workspace_bytes, void* stream);

/* get_time_evolution alone (I:855-896): writes time_dev[N] and u_dev[N][d][d]. */
int spinsim_time_evolution(const spinsim_plan* plan, const spinsim_field* field, double t0, double dt_int,
                           double dt_out, int64_t n_out, double* time_dev, double* u_dev, void* workspace_dev,
                           size_t workspace_bytes, void* stream);

/* get_state (I:1089-1111) as a parallel prefix scan, with get_spin (I:899-959) fused when spin_dev
 * is non-NULL.  psi0 is a host complex[d] array. */
size_t spinsim_state_workspace_size(int32_t dim, int64_t n_out);
int spinsim_state(int32_t dim, const double* u_dev, int64_t n_out, const double* psi0, double* state_dev,
                  double* spin_dev, void* workspace_dev, size_t workspace_bytes, void* stream);

/* spinsim_state without a workspace argument; no counterpart in the reference.  For callers that may
 * not allocate device memory (a plugin that only receives buffers from a host application owning
 * every allocation, or a loop that cannot afford cudaMalloc's device-wide synchronisation): the scan's
 * scratch is a fixed array inside this library (5 MiB, held on every GPU that loads the library
 * until exit).  At most spinsim_state_static_max_steps() output steps (262144); larger inputs are
 * rejected with SPINSIM_ERR_INVALID.  The first call on a device looks up the array's device address
 * (make it before any stream capture).  Calls share the array: calls whose work overlaps on the GPU
 * race and must be serialised by the caller.  Allocates nothing. */
int64_t spinsim_state_static_max_steps(void);
int spinsim_state_static(int32_t dim, const double* u_dev, int64_t n_out, const double* psi0, double* state_dev,
                         double* spin_dev, void* stream);

/* One evaluate() split into pieces of consecutive output steps (across launches or GPUs; no
 * counterpart in the reference, whose get_state I:1087-1111 is one serial loop).  For a piece with
 * operators u_dev[n][d][d] (computed with spinsim_instance.interval0 = the piece's first time index):
 *   spinsim_piece_product writes P = U[n-1] ... U[0] (complex [d][d]) to product_dev and leaves the
 *   piece's prefixes in the workspace (spinsim_state_workspace_size(dim, n) bytes);
 *   spinsim_piece_states, given psi_in = the state entering the piece (the pieces before it applied to
 *   psi0, in order), writes state[i] = U[i-1] ... U[0] psi_in and spin from the prefixes left in the
 *   same workspace by spinsim_piece_product on the same u_dev, and must follow it on the stream.
 * The state entering piece r is P_{r-1} ... P_0 psi0: one exchange of d x d products between pieces. */
int spinsim_piece_product(int32_t dim, const double* u_dev, int64_t n_out, double* product_dev, void* workspace_dev,
                          size_t workspace_bytes, void* stream);
int spinsim_piece_states(int32_t dim, const double* u_dev, int64_t n_out, const double* psi_in, double* state_dev,
                         double* spin_dev, void* workspace_dev, size_t workspace_bytes, void* stream);

/* Ensemble mean of the spin on the device (no counterpart in the reference, whose users average
 * Results.spin on the host after copying every member's states back): for members m = 0 .. members-1
 * whose spin series start at output step first + m * stride of spin_dev (e.g. the instances of a
 * batch with equal N: first = out_offset of the first, stride = N), mean_dev[i][c] = the average
 * over members of spin[first + m * stride + i][c], i < n_out.  The sum runs in a fixed order (chunks
 * of members, then the chunks in order).  Workspace: spinsim_spin_mean_workspace_size bytes. */
size_t spinsim_spin_mean_workspace_size(int32_t members, int64_t n_out);
int spinsim_spin_mean(const double* spin_dev, int64_t first, int64_t stride, int32_t members, int64_t n_out,
                      double* mean_dev, void* workspace_dev, size_t workspace_bytes, void* stream);

/* get_spin alone (I:899-959; spin_calculator I:961-988): spin_dev[N][3] from state_dev[N][d]. */
int spinsim_spin(int32_t dim, const double* state_dev, int64_t n_out, double* spin_dev, void* stream);

/* Batched evaluation (no counterpart in the reference, which runs one evaluate() per sweep): many
 * instances of possibly different spin, duration and step in one persistent launch.  prepare uploads
 * the descriptors and the longest-first tile queue into the workspace (stream-ordered) and returns a
 * handle; launch issues only kernel launches and a counter reset, so it can be captured into a CUDA
 * graph and replayed.  Outputs are the flat arrays addressed by the instances' offsets. */
/* Packs a batch's built-in fields (host only; no counterpart in the reference, whose samplers close
 * over their own arrays, I:1941-2147) into one host buffer for one copy to the device buffer at
 * device_base, and fills fields_out[n_fields] with device addresses.  Layout: eight table descriptors
 * per tabulated field first, then every field's arrays (times shared between channels once).  plan:
 * 8 int64 per row; per field a header {kind (1 tables, 2 tones), n_rows, bias (double[8]), gain
 * (double[8], or 0 for ones), tone rows, tone row doubles, int32 tone_start[8] + tone_count[8], 0}
 * followed, for tables, by n_rows channel rows {channel, time, amplitude, size, order, zero_boundary,
 * alias (-1 or the field-local index of an earlier channel with the same times), 0}; the pointers are
 * host addresses.  Returns the doubles written, or a negative error code. */
int64_t spinsim_pack_fields(int32_t n_fields, const int64_t* plan, int64_t n_plan_rows, double* host,
                            int64_t host_doubles, uint64_t device_base, spinsim_field* fields_out);

/* Batch descriptors from evaluate() arguments (host only): for each instance i the step
 * normalisation of I:1025-1034 (as spinsim_normalise_steps), its output offsets packed one after
 * another in the flat arrays, field index i and psi0 from psi0[6 i .. 6 i + 2 dim) (re, im
 * interleaved).  totals (optional) receives {output steps, U doubles, state doubles, integration
 * steps}.  The batched counterpart of the per-call set-up in evaluate (I:1025-1052). */
int spinsim_batch_describe(int32_t n, const double* t0, const double* t1, const double* dt_int, const double* dt_out,
                           const int32_t* dim, const double* psi0, spinsim_instance* out, int64_t* totals);

size_t spinsim_batch_workspace_size(const spinsim_plan* plan, const spinsim_instance* instances,
                                    int32_t n_instances, int32_t n_fields);
int spinsim_batch_prepare(const spinsim_plan* plan, const spinsim_instance* instances, int32_t n_instances,
                          const spinsim_field* fields, int32_t n_fields, void* workspace_dev,
                          size_t workspace_bytes, void* stream, spinsim_batch** out);

/* The same preparation with every descriptor written into host_staging (at least
 * spinsim_batch_staging_size bytes; page-locked for the copy to be asynchronous) and uploaded with
 * one copy on `stream`; host_staging must stay unchanged until that copy has completed.  The
 * descriptors lead the workspace, so the copy is one contiguous block. */
size_t spinsim_batch_staging_size(const spinsim_plan* plan, const spinsim_instance* instances, int32_t n_instances,
                                  int32_t n_fields);
int spinsim_batch_prepare_staged(const spinsim_plan* plan, const spinsim_instance* instances, int32_t n_instances,
                                 const spinsim_field* fields, int32_t n_fields, void* workspace_dev,
                                 size_t workspace_bytes, void* host_staging, size_t staging_bytes, void* stream,
                                 spinsim_batch** out);
int spinsim_batch_launch(const spinsim_batch* batch, double* time_dev, double* u_dev, double* state_dev,
                         double* spin_dev, void* stream);

/* Batches with an FP32-bulk plan: later launches write step_norms_dev[i] for every output step i of
 * the flat arrays (instances at their out_offset), as spinsim_evaluate_with_norms does; NULL stops it. */
int spinsim_batch_set_step_norms(spinsim_batch* batch, float* step_norms_dev);

/* The launch shape a prepared batch runs with (no counterpart in the reference): its tile queue,
 * the output steps per tile, the lanes per output step, and the state scan's tiles. */
typedef struct {
    int64_t tiles;          /* time-evolution tiles in the queue */
    int64_t scan_tiles;     /* state-scan tiles (with padding to whole warps) */
    int32_t lanes;          /* lanes per output step */
    int32_t tile_intervals; /* output steps per time-evolution tile */
    int32_t scan_partials;  /* 1: the time evolution writes the state scan's tile partials (tensor path,
                               every instance's field on it) and the scan launches no tile products */
    int32_t reserved;
} spinsim_batch_info;
int spinsim_batch_get_info(const spinsim_batch* batch, spinsim_batch_info* info);
int spinsim_batch_destroy(spinsim_batch* batch);

/* Diagnostics (no counterpart in the reference): one launch of an FMA-throughput loop that fills the
 * device (precision 0: FP64, 1: FP32).  *flops receives the operations it performs; time the launch
 * with events on `stream` to get the pipe's peak rate, the denominator of the kernels' roofline. */
int spinsim_fma_peak(int32_t precision, double* flops, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SPINSIM_B200_H */
