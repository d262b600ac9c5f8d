/* ses_gpu.h -- C ABI of the B200 split-operator (Strang) TDSE step.
 *
 * Drop-in boundary for the reference core's propagator / propagator-tables /
 * fft3 call surface (parkyere/ShoeridingerEquationSolver).  The reference has
 * no FFI layer of its own: callers use C++ module interfaces.  Each entry point
 * below names the reference interface it replaces (file:line inside the
 * reference project).  Plain pointers and sizes only; no exceptions cross
 * this boundary; every call returns a ses_status and, on failure, leaves a
 * message for ses_last_error() on the calling thread.
 *
 * Data conventions (same as the reference):
 *   - complex fields are interleaved (re, im) doubles on the host, flat
 *     x-fastest order, index i + nx*(j + ny*k)       (core/src/grid.ixx:20-30)
 *   - grids are periodic: spacing = (xmax - xmin)/n  (core/src/grid.ixx:4-18)
 *   - forward FFT unnormalised with e^{-}, inverse carries 1/N
 *                                                     (core/src/fft.ixx:14-18)
 *   - 2D scenes are Grid3D with nz = 1, 1D is nx x 1 x 1 (axes of length 1
 *     are left untransformed; wavenumber 0)           (core/src/spectral.ixx:14-23)
 *
 * Supported axis lengths: 2^a 3^b 5^c up to 4096 (the reference accepts powers
 * of two only and throws std::invalid_argument otherwise; here other lengths
 * return SES_EINVAL).
 *
 * Threading: calls on one handle must be serialised by the caller (like the
 * reference engine, vk_compute.ixx:272-274); distinct handles are independent.
 * All device work of a handle is ordered on that handle's CUDA stream.
 */
#ifndef SES_GPU_H
#define SES_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SES_API __attribute__((visibility("default")))
#else
#define SES_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ses_status {
    SES_OK = 0,
    SES_EINVAL = 1,     /* bad size, radix, pointer or argument */
    SES_ENOMEM = 2,     /* device allocation failed or memory budget exceeded */
    SES_ETIMEDOUT = 3,  /* a bounded wait expired */
    SES_EDEVICE = 4,    /* CUDA error; the handle should be destroyed */
    SES_EBUSY = 5,      /* resource busy (serving queue full) */
    SES_ENOTFOUND = 6   /* unknown request id */
} ses_status;

/* SES_C128: plain FP64 path (complex128 psi and tables).
 * SES_C64:  complex64 psi and FFT arithmetic; phase tables built in FP64,
 *           diagonal multiplies and all reductions in FP64. */
typedef enum ses_precision { SES_C128 = 0, SES_C64 = 1 } ses_precision;

/* Grid1D (core/src/grid.ixx:10-17) */
typedef struct ses_axis {
    double xmin;
    double xmax;
    int32_t n;
} ses_axis;

/* Grid3D (core/src/grid.ixx:22-30) */
typedef struct ses_grid_desc {
    ses_axis x, y, z;
} ses_grid_desc;

typedef struct ses_solver* ses_handle;

/* Observables of the resident psi at a step boundary, FP64 accumulation. */
typedef struct ses_observables {
    double norm;         /* sum |psi|^2 dV                        (core/src/field.ixx:68-74) */
    double energy;       /* <V> + <T>, each term normalised separately
                                                          (core/src/observables.ixx:202-234) */
    double energy_v;     /* sum V|psi|^2 / sum |psi|^2                                 */
    double energy_t;     /* sum k^2/(2m)|phi|^2 / sum |phi|^2, phi = FFT(psi)          */
    double p_range;      /* absolute sum |psi|^2 dV over cells with x in [xlo, xhi)
                                                          (core/src/observables.ixx:121-130,
                                                   scenario/src/tunneling_director.ixx:54-85) */
    double mean_pos[3];  /* (core/src/observables.ixx:134-153) */
    double sigma_pos[3]; /* (core/src/observables.ixx:155-178) */
    double mean_mom[3];  /* (core/src/observables.ixx:180-199) */
} ses_observables;

/* ---- library ---- */
SES_API const char* ses_version(void);
/* Message of the last failing call on this thread ("" when none). */
SES_API const char* ses_last_error(void);
SES_API ses_status ses_device_count(int* out);

/* ---- SplitOperator3D surface (core/src/propagator.ixx:68-134) ----
 * ses_gpu_create replaces SplitOperator3D(const Grid3D&, const std::vector<double>& V,
 * double dt, double mass = 1.0) (propagator.ixx:72-101) together with the
 * reference GPU Engine::initialize(ctx, grid, kernels, V, dt, psi0, mass)
 * (solver/src/vk_engine.ixx:173-580): it builds the FP64 phase tables on the
 * device and uploads psi0 (NULL -> zero field).  V has nx*ny*nz doubles.
 * SplitOperator1D (propagator.ixx:21-66) is the same call with ny = nz = 1
 * and mass = 1. */
SES_API ses_status ses_gpu_create(const ses_grid_desc* grid, ses_precision prec, double dt, double mass,
                          const double* V, const double* psi0, ses_handle* out);
/* ImaginaryTimePropagator3D(grid, V, dtau, mass) (core/src/imaginary_time.ixx:64-96) and the
 * GPU relax path (solver/src/vk_engine.ixx:1047-1080): the same handle with the real weights
 * exp(-V dtau/2) and exp(-k^2 dtau/(2m)) in place of the phase tables.  Step it with
 * ses_gpu_relax; ses_gpu_observe gives <H>.  Lines above 4096 points are not supported. */
SES_API ses_status ses_gpu_create_imag(const ses_grid_desc* grid, ses_precision prec, double dtau, double mass,
                                       const double* V, const double* psi0, ses_handle* out);
/* relax(Field3D&, nsteps) (imaginary_time.ixx:98-108): nsteps Strang steps of imaginary
 * time, psi renormalised to sum |psi|^2 dV = 1 on the device every renorm_every steps
 * (<= 0: every step, as the reference; the result differs only by rounding since the step
 * is linear).  energy (nullable): -ln(norm^2) / (2 r dtau) over the last r steps before
 * the final renormalisation, which converges to the ground-state energy; with energy
 * NULL the call only queues the work. */
SES_API ses_status ses_gpu_relax(ses_handle h, int nsteps, int renorm_every, double* energy);
/* Engine::destroy (vk_engine.ixx) */
SES_API ses_status ses_gpu_destroy(ses_handle h);
/* Engine::set_potential (vk_engine.ixx): rebuild the potential phase table. */
SES_API ses_status ses_gpu_set_potential(ses_handle h, const double* V);
/* Engine::set_absorber(mask) (vk_engine.ixx:880-941): real per-cell mask,
 * N doubles; NULL clears it.  A mask that is an exact product of per-axis
 * profiles (absorbing_mask, potential.ixx:216-233) is stored as three 1D
 * profiles; any other mask is stored in full. */
SES_API ses_status ses_gpu_set_absorber(ses_handle h, const double* mask);
/* Separable absorber: mask(i,j,k) = mx[i] * my[j] * mz[k]. */
SES_API ses_status ses_gpu_set_absorber_separable(ses_handle h, const double* mx, const double* my,
                                          const double* mz);
/* SplitOperator3D::step(Field3D&, int nsteps) (propagator.ixx:110-119) on the
 * resident psi; with absorb != 0 psi is multiplied by the mask after EVERY
 * step (Engine::step(n, absorb), vk_engine.ixx:597-636).  Interior half-kicks
 * are merged into full kicks, so psi is in real space only at batch ends.
 * Asynchronous: returns once the work is queued on the handle's stream. */
SES_API ses_status ses_gpu_step(ses_handle h, int nsteps, int absorb);
/* driven_step(psi, prop, DipoleDrive{axis, amplitude, omega}, t0, nsteps) (core/src/drive.ixx:50-65)
 * and Engine::driven_step (solver/src/vk_engine.ixx:836-876): each step is
 * kick(t) . Strang step . kick(t + dt), kick = psi * cis(-theta (axis . r)),
 * theta = amplitude cos(omega t) dt/2, t = t0 + s dt; absorb as in ses_gpu_step.
 * 2D and 3D grids.  The kick between two steps is applied as one phase. */
SES_API ses_status ses_gpu_step_driven(ses_handle h, int nsteps, int absorb, const double* axis, double amplitude,
                                       double omega, double t0);
/* fft(Field3D&) / ifft(Field3D&) (core/src/fft.ixx:102-188) on the resident
 * psi: direction 0 = forward (unnormalised), 1 = inverse (1/N). */
SES_API ses_status ses_gpu_fft3(ses_handle h, int direction);
/* half_potential_phase() / kinetic_phase() (propagator.ixx:103-108): the
 * full-N complex128 tables cis(-V dt/2) and cis(-(kx^2+ky^2+kz^2)/(2m) dt),
 * evaluated in FP64 on the device.  Either pointer may be NULL. */
SES_API ses_status ses_gpu_tables(ses_handle h, double* half_v, double* kin);
/* dt() (propagator.ixx:103) */
SES_API ses_status ses_gpu_dt(ses_handle h, double* dt);
/* norm_sq, mean_energy, probability_in_range, mean_position, sigma_position,
 * mean_momentum of the resident psi (observables.ixx:121-234), with xlo/xhi
 * the x-interval of p_range.  Blocks until the values are on the host. */
SES_API ses_status ses_gpu_observe(ses_handle h, double xlo, double xhi, ses_observables* out);
/* The same observables queued on the handle's stream (its batch's stream while
 * it is a member) without waiting, like Engine::step_async / wait_async
 * (solver/src/vk_engine.ixx:638-698): out receives them once the stream has
 * reached this point (ses_gpu_sync, ses_batch_sync, or an event the caller
 * records on that stream).  out should be page-locked host memory; the values
 * equal ses_gpu_observe's bit for bit. */
SES_API ses_status ses_gpu_observe_async(ses_handle h, double xlo, double xhi, ses_observables* out);
/* Engine::readback / upload_state (vk_engine.ixx:2136-2155, 1083-1089,
 * 2413-2421): interleaved complex128 host arrays of N elements (the C64 path
 * rounds on upload and widens on readback).  Both block until done. */
SES_API ses_status ses_gpu_read_psi(ses_handle h, double* psi_out);
SES_API ses_status ses_gpu_write_psi(ses_handle h, const double* psi_in);
/* psi snapshot wire format (the readback / upload_state layout of Engine,
 * solver/src/vk_engine.ixx:2136-2155, 2413-2421, with a header): 128-byte header
 * {"SESPSI1", precision, n[3], box[6], dt, mass, steps} then psi in the handle's own
 * precision, interleaved float (SES_C64) or double (SES_C128) pairs, x fastest, no
 * conversion.  For checkpoints and preemption.  Snapshot with out = NULL only
 * reports the size; restore checks precision and grid.  Both block. */
SES_API ses_status ses_gpu_snapshot(ses_handle h, int64_t steps, void* out, size_t cap, size_t* bytes);
SES_API ses_status ses_gpu_restore(ses_handle h, const void* snap, size_t bytes, int64_t* steps);
/* |psi|^2 (FP32) of the plane `index` along `axis` (0 x, 1 y, 2 z), the other two
 * axes in order (lower axis fastest): nx*ny floats for axis 2, and so on.  For
 * streaming density slices.  Blocks. */
SES_API ses_status ses_gpu_density_slice(ses_handle h, int axis, int index, float* out);
/* Wait for the handle's queued work; the wait is bounded by timeout_ms
 * (<= 0: 10 s, the reference's fence limit vk_compute.ixx:297-327) and
 * returns SES_ETIMEDOUT when it expires. */
SES_API ses_status ses_gpu_sync(ses_handle h, int timeout_ms);
/* Use an external cudaStream_t (NULL: the handle's own stream). */
SES_API ses_status ses_gpu_set_stream(ses_handle h, void* cuda_stream);
/* Device pointer and byte size of the resident psi (complex128 or complex64,
 * x-fastest), for callers that keep data on the device. */
SES_API ses_status ses_gpu_psi_device(ses_handle h, void** dptr, size_t* bytes);
/* Engine::profile_step (vk_engine.ixx:700-774): run an nsteps Strang batch
 * (absorb as in ses_gpu_step) launching every axis pass directly, with a CUDA
 * event pair around each launch on the handle's stream.  pass_ms[8] receives
 * the mean milliseconds per launch of:
 *   [0] x pass between steps   [1] y forward   [2] last-axis fused (fwd, K/N, inv)
 *   [3] y inverse              [4] x pass at batch start   [5] x pass at batch end
 *   [6] total batch (first to last event)   [7] number of launches
 * Unused kinds report 0.  psi advances exactly as with ses_gpu_step.  Blocks. */
SES_API ses_status ses_gpu_profile_step(ses_handle h, int nsteps, int absorb, double* pass_ms);
/* Tile-shape autotuner (plays the role of the reference's VkFFT plan set-up,
 * solver/src/vk_engine.ixx:3220-3306): times every compiled tile variant of
 * each axis pass (tile width, ring depth, warps per CTA, register budget) and
 * the register-path kernels on the handle's scratch field -- psi is not
 * touched -- and keeps the fastest per axis.  flags bit 0: also record the
 * choice in the on-disk cache ($SES_TUNE_CACHE, default
 * ~/.cache/ses_b200/autotune.txt), which later handles of the same shape read
 * at creation.  Blocks. */
SES_API ses_status ses_gpu_autotune(ses_handle h, int flags);
/* Human-readable description of the handle's axis plans and chosen variants. */
SES_API ses_status ses_gpu_plan_info(ses_handle h, char* buf, size_t len);
/* Device bytes held by the handle. */
SES_API ses_status ses_gpu_footprint(ses_handle h, size_t* bytes);
/* Failure-detection hook, the counterpart of the reference's 10 s fence timeout
 * that marks the engine device_lost (solver/src/vk_compute.ixx:297-327): every
 * wait inside this handle's pipelined (TMA-fed) passes is bounded by
 * wait_cycles SM clock cycles (0: about 2 s, the default), and with
 * extra_tx_bytes > 0 every tile's barrier expects that many bytes more than its
 * copies deliver, so its wait runs out -- the pass then records the error,
 * drains its copies (bounded) and returns, no load or store is changed, and the
 * next ses_gpu_sync reports SES_ETIMEDOUT with the context still usable.  For
 * tests of that path; (0, 0) restores normal operation.  Waits for queued work
 * first; extra_tx_bytes <= 4096. */
SES_API ses_status ses_gpu_set_wait_limit(ses_handle h, int64_t wait_cycles, uint32_t extra_tx_bytes);
/* Engine::norm_and_peak (solver/src/vk_engine.ixx:1665-1692, shader
 * solver/shaders/norm_peak.comp.slang): norm = sum |psi|^2 dV and peak =
 * max |psi|^2 of the resident psi, FP64 sums folded in a fixed order
 * (deterministic).  Either output may be NULL.  Blocks. */
SES_API ses_status ses_gpu_norm_and_peak(ses_handle h, double* norm, double* peak);
/* Engine::scale(s) (solver/src/vk_engine.ixx:2120-2133, shader
 * solver/shaders/scale.comp.slang:12-19): psi <- factor * psi, the directors'
 * drift renormalisation (scenario/src/base_director.ixx:340-352).  Queued on
 * the handle's stream. */
SES_API ses_status ses_gpu_scale(ses_handle h, double factor);
/* Records the handle's step graph ahead of the first long step batch (the
 * reference engine records its command buffers in Engine::initialize,
 * solver/src/vk_engine.ixx:173-580), so that no capture happens inside a
 * caller's timed or latency-critical region.  absorb selects the graph with or
 * without the mask; psi is not touched. */
SES_API ses_status ses_gpu_prepare(ses_handle h, int absorb);

/* ---- allocation-free entry point ----
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory -- a host framework whose caching allocator already owns the GPU's
 * memory, where a cudaMalloc from this library could fail, or a loop that
 * must not pay cudaMalloc/cudaFree synchronisation: the real-space
 * observables of a caller-owned device field, with no handle and no device
 * allocation of any kind.
 *   psi_dev  nx*ny*nz complex128 (SES_C128) or complex64 (SES_C64) values, x-fastest
 *   V_dev    nx*ny*nz doubles, or NULL (then out[1] = 0)
 *   out_dev  9 doubles in device memory: norm, <V>, probability in [xlo, xhi),
 *            mean position x y z, sigma x y z (same definitions as ses_gpu_observe)
 *   cuda_stream  the stream to run on (NULL: the default stream); the call
 *            returns once the work is queued
 * Scratch is a fixed 2.25 MiB array in the library's device image, held by
 * every GPU that loads the library until the process exits, so grids are
 * limited to 2^27 points (512^3): larger grids return SES_EINVAL.  All calls
 * on a device share that array: calls that overlap on the GPU (different
 * streams, or different host threads) race and must be serialised by the
 * caller.  The first call on each device resolves the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture. */
SES_API ses_status ses_observe_real_noalloc(const ses_grid_desc* grid, ses_precision prec,
                                            const void* psi_dev, const double* V_dev, double xlo,
                                            double xhi, double* out_dev, void* cuda_stream);

/* ---- batches: many independent propagations per launch ----
 * The reference advances one field per Engine (solver/src/vk_engine.ixx:
 * 597-698) and batches sweeps on the CPU by parallel_for over instances
 * (core/src/parallel.ixx:195-238); a batch replaces that loop.  Handles join a
 * batch; members with the same grid shape and precision form a class, and each
 * axis pass of a step is ONE launch per class whose CTAs walk instance x
 * line tiles.  Classes run concurrently on their own streams; interior steps
 * are CUDA graphs.  Every member keeps its own field, potential table, axis
 * tables, dt, mass and absorber, and computes exactly what ses_gpu_step would
 * with the same step batching.  Shapes without batched kernels step member by
 * member.  A member's stream is the batch's stream while it belongs to it;
 * calls on a member (observe, read_psi, ...) stay valid and are ordered after
 * the batch's queued steps.  Destroying a member removes it first.  A batch
 * is single-threaded like a handle. */
typedef struct ses_batch_s* ses_batch;
SES_API ses_status ses_batch_create(ses_batch* out);
SES_API ses_status ses_batch_destroy(ses_batch b);
/* SES_EBUSY if h already belongs to a batch; waits for h's queued work. */
SES_API ses_status ses_batch_add(ses_batch b, ses_handle h);
SES_API ses_status ses_batch_remove(ses_batch b, ses_handle h);
/* Every member advances nsteps merged Strang steps (absorb: members that have an
 * absorber apply it after every step).  Returns once the work is queued; the
 * first call after a membership change waits for queued work and uploads the
 * per-member pass arguments. */
SES_API ses_status ses_batch_step(ses_batch b, int nsteps, int absorb);
/* ses_gpu_prepare for every class of the batch (its per-class step graph). */
SES_API ses_status ses_batch_prepare(ses_batch b, int absorb);
/* ses_gpu_observe of every member, in the order they were added (count must be
 * the member count), with one wait for the whole batch. */
SES_API ses_status ses_batch_observe(ses_batch b, double xlo, double xhi, ses_observables* out, int count);
/* One round trip of every member with host buffers, as upload_state -> step
 * batch -> observables -> readback of the reference Engine (vk_engine.ixx:
 * 1083-1089, 597-698, 2136-2155) for each instance: psi_in[i] / psi_out[i]
 * are interleaved complex128 host arrays of member i (null entries skip that
 * member's upload or readback; null arrays skip all), obs (nullable) receives
 * ses_gpu_observe(xlo, xhi) after the steps, members in the order they were
 * added (count must be the member count).  Each class's uploads, steps,
 * observables and readbacks are queued on its own stream, largest class
 * first, so one class's PCIe transfers overlap the other classes' steps; the
 * results equal write_psi + ses_batch_step + observe + read_psi.  Host arrays
 * should be page-locked (cudaHostAlloc / pinned tensors): pageable memory
 * works but its copies do not overlap.  Blocks until done or timeout_ms
 * (<= 0: 60 s) has passed (SES_ETIMEDOUT). */
SES_API ses_status ses_batch_run(ses_batch b, const double* const* psi_in, int nsteps, int absorb, double xlo,
                                 double xhi, ses_observables* obs, double* const* psi_out, int count,
                                 int timeout_ms);
/* The same for the listed members only, each with its own x-interval. */
SES_API ses_status ses_batch_observe_some(ses_batch b, const ses_handle* hs, int count, const double* xlo,
                                          const double* xhi, ses_observables* out);
SES_API ses_status ses_batch_sync(ses_batch b, int timeout_ms);
SES_API ses_status ses_batch_set_stream(ses_batch b, void* cuda_stream);
SES_API ses_status ses_batch_members(ses_batch b, int* members, int* classes);
/* Per class (in order of first appearance), 5 values: mean milliseconds per
 * launch of the x pass between steps, the strided passes 1..3 of the step, and
 * their sum (one interior step of the whole class), timed with events around
 * nsteps interior steps run class after class on the batch stream.  Members
 * advance by a complete Strang batch of nsteps + 1 steps (nsteps + 2 for 1D).
 * Blocks. */
SES_API ses_status ses_batch_profile(ses_batch b, int nsteps, int absorb, double* ms, int count);
/* Tile-shape autotuner for every class: times the register-path and each
 * pipelined variant of the x pass and of each strided pass on the members'
 * scratch fields (psi is not touched) and keeps the fastest for the batch.
 * flags bit 0: also record the choice in the on-disk cache (as
 * ses_gpu_autotune), which later batches with a class of the same shape read.
 * Blocks. */
SES_API ses_status ses_batch_autotune(ses_batch b, int flags);
/* One line per class: shape, precision, members and the kernel of each pass. */
SES_API ses_status ses_batch_info(ses_batch b, char* buf, size_t len);

/* ---- serving: continuous batching of solve requests ----
 * No direct counterpart in the reference, whose directors run one scene per
 * Engine (solver/src/vk_engine.ixx:597-698, scenario/src/base_director.ixx)
 * and whose sweeps loop over instances on the CPU.  A server owns one batch
 * and a worker thread.  Requests are admitted first come, first served while
 * their estimated device bytes fit the budget; admitted fields and tables
 * stay resident in HBM.  All running requests advance together in rounds that
 * end at the earliest observation point or completion of any of them; new
 * requests join and finished ones leave between rounds.  Observables
 * (ses_gpu_observe) are recorded every observe_every steps and at
 * completion; latency is submission to completion.  Every call is
 * thread-safe. */
typedef struct ses_server_s* ses_server;

typedef struct ses_request {
    ses_grid_desc grid;
    ses_precision prec;
    double dt, mass;            /* mass <= 0 means 1 */
    const double* V;            /* nx*ny*nz doubles, copied at submit */
    const double* psi0;         /* nx*ny*nz interleaved complex128, copied at submit */
    const double* mask_x;       /* separable absorber profiles (nx, ny, nz doubles), */
    const double* mask_y;       /* applied after every step; all three or none */
    const double* mask_z;
    int32_t nsteps;             /* >= 1 */
    int32_t observe_every;      /* 0: observe at completion only */
    double xlo, xhi;            /* interval of ses_observables.p_range */
} ses_request;

typedef struct ses_record {
    int64_t id;
    int32_t step;               /* steps completed when observed */
    int32_t final_record;       /* 1 on the record taken at completion */
    double t_ms;                /* since submission */
    ses_observables obs;
} ses_record;

enum { SES_REQ_QUEUED = 0, SES_REQ_RUNNING = 1, SES_REQ_DONE = 2, SES_REQ_CANCELLED = 3, SES_REQ_FAILED = 4 };

typedef struct ses_serve_stats_t {
    int64_t submitted, admitted, completed, cancelled, failed, queued, running, rounds;
    size_t bytes_in_use, budget;
    double gridpt_steps;        /* grid points x steps advanced by all rounds */
    double busy_ms;             /* wall time spent in rounds */
    double wall_ms;             /* since open */
    double latency_p50_ms, latency_p99_ms;  /* over completed requests */
} ses_serve_stats_t;

/* max_round_steps: longest round (0: 100). */
SES_API ses_status ses_serve_open(size_t budget_bytes, int max_round_steps, ses_server* out);
/* Copies the request's arrays; SES_ENOMEM if it can never fit the budget. */
SES_API ses_status ses_serve_submit(ses_server s, const ses_request* r, int64_t* id);
/* Moves up to cap pending records of request id into recs; *state = SES_REQ_*. */
SES_API ses_status ses_serve_poll(ses_server s, int64_t id, ses_record* recs, int cap, int* n, int* state);
/* After SES_REQ_DONE: the final psi (interleaved complex128, once) and the latency. */
SES_API ses_status ses_serve_result(ses_server s, int64_t id, double* psi_out, double* latency_ms);
SES_API ses_status ses_serve_cancel(ses_server s, int64_t id);
/* Waits (bounded) until every submitted request has finished. */
SES_API ses_status ses_serve_wait_idle(ses_server s, int timeout_ms);
SES_API ses_status ses_serve_stats(ses_server s, ses_serve_stats_t* out);
/* Cancels whatever is still queued or running, joins the worker, frees everything. */
SES_API ses_status ses_serve_close(ses_server s);

/* ---- fft surface on host arrays (core/src/fft.ixx:75-188) ----
 * fft(std::vector<cd>&) / ifft(...) and fft(Field3D&) / ifft(Field3D&):
 * n[3] = (nx, ny, nz), data = interleaved complex128, transformed in place
 * through the device. */
SES_API ses_status ses_fft3_host(const int32_t* n, ses_precision prec, double* data, int inverse);

#ifdef __cplusplus
}
#endif
#endif /* SES_GPU_H */
