/*
 * sodecl_cuda.h -- C ABI of libsodecl_cuda.so, the B200 (sm_100a) engine for
 * SODECL's fixed-step integrators.
 *
 * Plain C types only: every caller (the C++ sodecl::sodeclmgr, the Python
 * module sodecl_interface, ctypes, cgo, ...) binds the same entry points.
 *
 * Life cycle, mirroring the reference's sodeclmgr (src/sodeclmgr.cpp):
 *
 *   sodecl_cfg_init(&cfg); ...fill cfg...      ctor              :26-83
 *   sodecl_cuda_create(&cfg, &ctx)             choose_device     :164
 *   sodecl_cuda_compile(ctx, src, len)         create_kernel_string + build_program
 *                                                                :374-503, :559-622
 *   sodecl_cuda_upload(ctx, t0, y0, p, cnt)    set_t0/y0/params + create/write_buffers
 *                                                                :654-829
 *   sodecl_cuda_run(ctx, out, len)             run_sode_solver   :921-1035
 *   sodecl_cuda_destroy(ctx)                   ~sodeclmgr        :88-148
 *
 * Status codes: SODECL_OK (0) on success, a negative SODECL_ERR_* otherwise;
 * sodecl_cuda_last_error() then holds a message.  (The C++ sodeclmgr maps
 * them to the reference's 1 = success / 0 = failure.)
 *
 * Ownership: the library owns all device memory it allocates; the caller owns
 * every host array and every pointer it passes in.  Threading: a context is
 * used by one host thread at a time; distinct contexts are independent.
 */
#ifndef SODECL_CUDA_H
#define SODECL_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 4: sodecl_cfg gained record_store (after max_steps) */
#define SODECL_CUDA_ABI_VERSION 4

/* status codes */
#define SODECL_OK 0
#define SODECL_ERR_INVALID_ARG (-1)   /* a size, pointer or option is out of range */
#define SODECL_ERR_COMPILE (-2)       /* NVRTC rejected the program; see the build log */
#define SODECL_ERR_CUDA (-3)          /* a CUDA runtime call failed */
#define SODECL_ERR_NO_DEVICE (-4)     /* no CUDA device, or the ordinal does not exist */
#define SODECL_ERR_STATE (-5)         /* called out of order (e.g. run before upload) */
#define SODECL_ERR_NO_JACOBIAN (-6)   /* implicit solver, system file has no calc_jacobian */
#define SODECL_ERR_NO_STOCH (-7)      /* stochastic solver, system file has no sode_system_stoch */
#define SODECL_ERR_OUT_OF_MEMORY (-8) /* a device or pinned-host allocation failed */
#define SODECL_ERR_UNSUPPORTED (-9)   /* not available in this build / on this device */

/* solver numbering of the reference's solver_Type (include/solver_Type.hpp:14-20) */
#define SODECL_STOCHASTIC_EULER 0
#define SODECL_EULER 1
#define SODECL_RUNGE_KUTTA 2
#define SODECL_IMPLICIT_EULER 3
#define SODECL_IMPLICIT_MIDPOINT 4
/* No counterpart in the reference (its README lists variable-step solvers as
 * future work): Dormand-Prince 5(4) with adaptive steps per orbit.  Records
 * land on the same grid as the fixed-step solvers (every kernel_steps * dt);
 * dt is the first step tried; rtol, atol and max_steps below control it.
 * One thread per orbit; not in batches or the adjoint. */
#define SODECL_DORMAND_PRINCE 5

#define SODECL_FP64 0
#define SODECL_FP32 1

/* how programs divide: SODECL_DIV_RECIPROCAL computes a/b as a*r plus two FMA
 * corrections with r = 1/b (hoistable out of the step loop for parameters and
 * constants), returns NaN at once for a NaN operand, and falls back to IEEE
 * division outside [2^-500, 2^500) (FP32: [2^-60, 2^60)): the same quotient as
 * SODECL_DIV_IEEE bit for bit (NaN payloads aside).  SODECL_DIV_DEFAULT (what
 * sodecl_cfg_init sets) is the reciprocal form in FP64 and IEEE division in
 * FP32 and for the adaptive solver.  On the oculomotor RK4 workload in FP64 the reciprocal form is 2 %
 * faster on converging orbits and 1.8x on diverged ones; in FP32 it gains on
 * diverged orbits and loses on converging ones.  sodecl_cuda_autotune measures
 * both for a given system file. */
#define SODECL_DIV_RECIPROCAL 0
#define SODECL_DIV_IEEE 1
#define SODECL_DIV_DEFAULT 2

/* per-orbit status flags (sodecl_cuda_status) */
#define SODECL_FLAG_NEWTON_CAP 1   /* some implicit step stopped at newton_max_iter, or an
                                      adaptive record interval ran out of max_steps or of
                                      representable step sizes (its state is then NaN) */
#define SODECL_FLAG_NONFINITE 2    /* a stored record held NaN or Inf */

typedef struct sodecl_ctx sodecl_ctx;

/* Run configuration: the reference's constructor arguments
 * (include/sodeclmgr.hpp:122-124) plus this library's options. */
typedef struct sodecl_cfg {
    int32_t solver;          /* SODECL_STOCHASTIC_EULER .. SODECL_DORMAND_PRINCE */
    double dt;               /* step; the program steps with dt printed to 6 significant
                                digits, as the reference's #define _m_dt_ does */
    double int_time;         /* tspan: records = count(j < int_time/(dt*kernel_steps)) + 1 */
    int32_t kernel_steps;    /* steps between records (reference: steps per launch) */
    int32_t num_equat;
    int32_t num_params;
    int32_t num_noi;         /* noise processes; > 0 only with the stochastic solver */
    int64_t list_size;       /* orbits */
    int32_t device;          /* CUDA device ordinal */
    int32_t local_group_size;/* threads per block; 0 = library default */
    int32_t precision;       /* SODECL_FP64 (default) or SODECL_FP32 */
    int32_t fmad;            /* 1 (default): allow FMA contraction; 0: exact IEEE op order */
    double newton_tol;       /* implicit solvers' residual bound; default 1e-7 (sodeclmgr.cpp:425) */
    int32_t newton_max_iter; /* implicit solvers' pass limit; default 1000 (ie.cl:69, im.cl:65) */
    int32_t record_f32;      /* device-API records stored as float (sodecl_cuda_launch only) */
    int32_t min_blocks_per_sm; /* launch-bounds occupancy hint for the compiler; 0 = default: none, except
                                  with one thread per orbit for the implicit and adaptive solvers,
                                  which are held to 128 registers a thread, and for FP64 RK4 on up to
                                  8 equations, held to 85 (1 lifts either) */
    int32_t division;        /* quotients: SODECL_DIV_DEFAULT (the default: reciprocal in FP64, IEEE in
                                FP32 and for SODECL_DORMAND_PRINCE), SODECL_DIV_RECIPROCAL or
                                SODECL_DIV_IEEE;
                                both give the IEEE-rounded quotient bit for bit */
    int32_t lanes_per_orbit; /* 0 or 1 (default): one thread per orbit.  2, 4, 8, 16 or 32:
                                that many lanes of a warp share an orbit, each evaluating
                                some of its equations (wide systems).  Needs the system
                                file's sode_system_row (and sode_system_stoch_row for the
                                stochastic solver); Euler, RK4 and Euler-Maruyama only.
                                Same results either way.  No counterpart in the reference. */
    double rtol;             /* SODECL_DORMAND_PRINCE: relative and absolute error per step, */
    double atol;             /*   err_i / (atol + rtol max(|y_i|, |y5_i|)) in RMS <= 1; default 1e-6, 1e-9 */
    int32_t max_steps;       /* SODECL_DORMAND_PRINCE: step attempts per record interval; default 100000 */
    int32_t record_store;    /* how one thread per orbit writes its records: SODECL_STORE_DIRECT
                                (default; one 8-byte store per equation, coalesced across the
                                warp) or SODECL_STORE_PAIRS (neighbouring orbits swap values
                                with a shuffle and each writes one equation of both as a
                                16-byte store).  Same records either way; the tuner times both.
                                One thread per orbit with the Euler, RK4 and Euler-Maruyama
                                solvers only (elsewhere the direct stores run).  No
                                counterpart in the reference. */
} sodecl_cfg;

#define SODECL_STORE_DIRECT 0
#define SODECL_STORE_PAIRS 1

/* Fills the defaults: Euler, fp64, fmad on, Newton 1e-7 / 1000, device 0,
 * SODECL_DIV_DEFAULT division, one thread per orbit, direct record stores,
 * rtol 1e-6, atol 1e-9, 100000 adaptive steps per record interval. */
void sodecl_cfg_init(sodecl_cfg *cfg);

/* Validates cfg and makes a context bound to cfg->device.  Needs no GPU
 * until upload.  Replaces sodeclmgr::sodeclmgr + choose_device
 * (src/sodeclmgr.cpp:26-83, :164). */
int sodecl_cuda_create(const sodecl_cfg *cfg, sodecl_ctx **out);

/* Builds the program for the user's system file (OpenCL C text, as the
 * reference reads it from disk) with NVRTC for sm_100a.  Needs no GPU.
 * Replaces create_kernel_string/create_program/build_program
 * (src/sodeclmgr.cpp:374-622). */
int sodecl_cuda_compile(sodecl_ctx *ctx, const char *system_src, size_t len);

/* Copies the initial state to the device: t0[list_size], y0[list_size][num_equat],
 * params[list_size][num_params] (orbit-major, as the reference's host arrays),
 * counters[list_size] the noise draw counters (stochastic solver; NULL draws
 * them as the reference does, U(-1e11, 1e11), from a generator seeded with 0).
 * For SODECL_DORMAND_PRINCE the same array holds each orbit's next step size
 * (NULL or values <= 0: start with dt), kept across runs and launches so that
 * results do not depend on how a run is split.
 * Replaces set_t0/set_y0/set_params + create_buffers/write_buffers
 * (src/sodeclmgr.cpp:654-829, counters :48-59). */
int sodecl_cuda_upload(sodecl_ctx *ctx, const double *t0, const double *y0, const double *params,
                       const double *counters);

/* Records one run produces: launches + 1 (src/sodeclmgr.cpp:951, :998). */
int64_t sodecl_cuda_num_records(const sodecl_ctx *ctx);

/* Integrates every orbit over int_time from the current device state and
 * writes num_records() records of num_equat x list_size doubles to `out` in
 * the reference's [record][equation][orbit] order (src/sodeclmgr.cpp:980-994).
 * `out` may be host memory (pageable or pinned) or device memory; NULL
 * discards the records (output_Type::None).  out_len is the capacity in
 * doubles.  The state stays on the device, so a second call continues from
 * where the first stopped.  Replaces run_sode_solver (:921-1035). */
int sodecl_cuda_run(sodecl_ctx *ctx, double *out, int64_t out_len);

/* Copies the current state back: any pointer may be NULL. */
int sodecl_cuda_download_state(sodecl_ctx *ctx, double *t, double *y, double *counters);

/* Per-orbit status accumulated since upload: Newton passes taken (accepted
 * steps for SODECL_DORMAND_PRINCE) and SODECL_FLAG_* bits.  Either pointer may be NULL.  (No counterpart in the
 * reference, which reports nothing per orbit.) */
int sodecl_cuda_status(sodecl_ctx *ctx, int64_t *newton_passes, int32_t *flags);

/* Device time of the last run's kernels in milliseconds (CUDA events). */
int sodecl_cuda_last_run_ms(const sodecl_ctx *ctx, double *kernel_ms, double *total_ms);

/* Copies the last error message / the NVRTC build log (NUL-terminated,
 * truncated to n bytes).  Return the full length. */
size_t sodecl_cuda_last_error(const sodecl_ctx *ctx, char *buf, size_t n);
size_t sodecl_cuda_build_log(const sodecl_ctx *ctx, char *buf, size_t n);

/* The generated program text (for debugging; the reference writes it to
 * Generated_kernel.cl, src/sodeclmgr.cpp:498-500). */
size_t sodecl_cuda_program_source(const sodecl_ctx *ctx, char *buf, size_t n);

void sodecl_cuda_destroy(sodecl_ctx *ctx);

const char *sodecl_cuda_strerror(int status);
int sodecl_cuda_abi_version(void);
int sodecl_cuda_device_count(int *count);
/* The device's name and compute capability ("NVIDIA B200", 10, 0); the name
 * is copied NUL-terminated into buf (up to n bytes; buf may be NULL).  For the
 * manager's log file; the reference's choose_device logs its OpenCL
 * device's name and version (src/sodeclmgr.cpp:195-205). */
int sodecl_cuda_device_describe(int device, char *buf, size_t n, int *major, int *minor);

/* ---- device-buffer path (torch / custom callers; no host copies) ------- */

/* One launch over caller-owned device buffers, on the caller's stream
 * (NULL = the legacy default stream).  Pointers are device pointers:
 * t[n], y[n][neq], params[n][npar] (doubles, in/out except params),
 * counters[n] (stochastic solver; step sizes for SODECL_DORMAND_PRINCE,
 * nullable there), records = base of a window
 * [record][neq][rec_stride] of double (or float with cfg.record_f32) whose
 * first row is record rec_first.  Runs record intervals
 * [chunk_begin, chunk_end), storing each interval's starting state, and the
 * final state as record chunk_end if write_final.  newton_passes/flags
 * (nullable) accumulate.  The context must be compiled; no upload needed.
 * Every buffer must be memory the context's device can access (its own
 * device memory, managed memory or pinned host memory): anything else, such
 * as a pageable host array, is refused with SODECL_ERR_INVALID_ARG before
 * any launch. */
typedef struct sodecl_launch {
    double *t;
    double *y;
    const double *params;
    double *counters;
    void *records;
    int64_t n;
    int64_t orbit_offset;   /* global orbit index of orbit 0 (noise stream) */
    int64_t rec_stride;
    int64_t rec_col0;
    int32_t chunk_begin;
    int32_t chunk_end;
    int32_t rec_first;
    int32_t write_final;
    int64_t *newton_passes;
    int32_t *flags;
} sodecl_launch;

int sodecl_cuda_launch(sodecl_ctx *ctx, const sodecl_launch *launch, void *stream);

/* ---- discrete adjoint (model fitting) -----------------------------------
 *
 * For every orbit, the mean squared error of its records against targets,
 *   loss_i = sum_{r,e} (y_{r,e,i} - target_{r,e,i})^2 / (records * num_equat),
 * and (optionally) its gradient with respect to the orbit's parameters and
 * initial state, by the discrete adjoint of the steps (FP64): of the Euler
 * and RK4 arithmetic, and of the implicit Euler / midpoint steps taken as
 * solved exactly (a transposed solve with calc_jacobian's full matrix per
 * step; the forward Newton passes stop at newton_tol, so the gradient is that
 * of the exact implicit step, closer the tighter the tolerance).  The
 * vector-Jacobian products come from the system file's calc_vjp, else its
 * calc_jacobian + calc_jacobian_params, else the right-hand side
 * differentiated in reverse mode (the system file compiled a second time
 * with a recording `double`).  The state is checkpointed every `ckpt_every`
 * steps and recomputed per segment; with ckpt_every >= steps the forward
 * sweep records the whole trajectory (steps x (4 num_equat + 1) doubles per
 * orbit for RK4, num_equat + 1 otherwise) and nothing is recomputed.  The
 * default picks that when the buffer takes at most half the free device
 * memory, else ~sqrt(steps).  The context keeps the buffer for its next call
 * (sodecl_cuda_release_scratch or sodecl_cuda_destroy frees it).  Gradients
 * are the same bit for bit with any spacing.
 * Records, steps and the step size follow the context's configuration; all
 * pointers are device pointers (checked as for sodecl_cuda_launch); the
 * launch goes on `stream`.  No counterpart in the reference. */
typedef struct sodecl_adjoint_io {
    const double *t0;       /* [n] */
    const double *y0;       /* [n][num_equat] */
    const double *params;   /* [n][num_params] */
    const double *targets;  /* [records][num_equat][n] */
    double *loss;           /* [n] out */
    double *grad_params;    /* [n][num_params] out, or NULL for the loss alone */
    double *grad_y0;        /* [n][num_equat] out, or NULL */
    int32_t *flags;         /* [n] out, or NULL: 4 = tape overflow (raise tape_entries),
                               1 = a Newton step stopped at newton_max_iter */
    int64_t n;              /* orbits, <= list_size */
    int32_t ckpt_every;     /* steps per checkpoint; 0 = the whole trajectory when it fits in half the
                               free device memory, else ceil(sqrt(steps)) */
    int32_t tape_entries;   /* operations one right-hand side may record; 0 = 256 */
    int32_t use_tape;       /* 1: differentiate sode_system on the tape even when the system file
                               provides the products itself -- calc_vjp(t, y, v, ybar, pbar, p)
                               (ybar += v^T df/dy, pbar += v^T df/dp), else calc_jacobian with
                               calc_jacobian_params (df/dp): optional additions to the
                               system-file interface, used in that order otherwise */
} sodecl_adjoint_io;

#define SODECL_FLAG_TAPE_OVERFLOW 4

int sodecl_cuda_adjoint(sodecl_ctx *ctx, const sodecl_adjoint_io *io, void *stream);

/* Kernel resources of the compiled program on its device (registers per
 * thread, local memory bytes per thread, max threads per block).  Needs a GPU. */
int sodecl_cuda_kernel_info(sodecl_ctx *ctx, int *regs, int *local_bytes, int *max_threads);

/* Autotuner: times candidate launch shapes (threads per block, resident-block
 * hints, and lanes per orbit when the system file has sode_system_row and the
 * solver is explicit or stochastic) and division modes on copies of the
 * first `sample_orbits` uploaded orbits for `sample_steps` steps, records
 * included -- the context's state does not advance -- then the winner with
 * paired record stores (SODECL_STORE_PAIRS), and rebuilds the program with
 * the fastest.  All candidates give identical results.  Writes the choice (any
 * pointer may be NULL; the store form is in the configuration,
 * sodecl_cuda_get_cfg). */
int sodecl_cuda_autotune(sodecl_ctx *ctx, int64_t sample_orbits, int32_t sample_steps, int32_t *block,
                         int32_t *min_blocks, int32_t *division, int32_t *lanes, double *best_ms);

/* Frees the device scratch a context keeps for its next call: the record
 * buffer of runs into host memory and the adjoint's checkpoint / trajectory
 * buffer (tens of GB for large fits), and the record buffer that destroyed
 * contexts left on its device (below).  The next call allocates again.  Waits
 * for the context's queued work.  No counterpart in the reference. */
int sodecl_cuda_release_scratch(sodecl_ctx *ctx);

/* A destroyed context leaves its record buffer (runs into host memory) to
 * the next context on the same device, one buffer per device, because the
 * reference's callers make a new manager for every call and a multi-GB
 * free and allocation per call cost up to hundreds of milliseconds.  This
 * frees it.  Call it before cudaDeviceReset.  No counterpart in the
 * reference. */
int sodecl_cuda_release_cached(int device);

/* The context's configuration as it stands, e.g. after sodecl_cuda_autotune. */
int sodecl_cuda_get_cfg(const sodecl_ctx *ctx, sodecl_cfg *cfg);

/* Division mode the program was actually built with (SODECL_DIV_*): the
 * reciprocal mode falls back to IEEE for system files that need plain double. */
int sodecl_cuda_program_division(const sodecl_ctx *ctx);

/* ---- heterogeneous batches ----------------------------------------------
 *
 * Many orbits of up to 32 classes -- each class a system file with a solver,
 * sizes and step -- and each orbit with its own step count, integrated by one
 * persistent kernel that takes orbits from per-class device work queues
 * (orbits sorted by decreasing step count, lanes refilled as their orbit
 * finishes), launched through a captured CUDA graph.  Final states only.
 * No counterpart in the reference, which integrates one system, one solver
 * and one step count per call (src/sodeclmgr.cpp:921-1035). */
typedef struct sodecl_batch sodecl_batch;

typedef struct sodecl_class_cfg {
    int32_t solver;
    int32_t num_equat;
    int32_t num_params;
    int32_t num_noi;
    double dt;               /* step, printed to 6 significant digits like _m_dt_ */
    double newton_tol;       /* default 1e-7 */
    int32_t newton_max_iter; /* default 1000 */
    int32_t lanes_per_orbit; /* 0 (default): automatic -- several lanes per orbit for classes of
                                12 or more equations whose system file has the per-row functions
                                (see sodecl_cfg.lanes_per_orbit), else one; 1: one lane;
                                2..32, a power of two: that many */
} sodecl_class_cfg;

void sodecl_class_cfg_init(sodecl_class_cfg *cfg);
int sodecl_batch_create(int device, int fmad, int division, sodecl_batch **out);
/* Adds a class (before compile); writes its id. */
int sodecl_batch_add_class(sodecl_batch *b, const char *system_src, size_t len, const sodecl_class_cfg *cfg,
                           int32_t *class_id);
/* Builds one NVRTC program with every class and the persistent kernel. */
int sodecl_batch_compile(sodecl_batch *b);
/* n orbits: class, step count, t0; y0 and params packed in orbit order with
 * each orbit's class widths; counters (NULL unless a class is stochastic). */
int sodecl_batch_set_items(sodecl_batch *b, int64_t n, const int32_t *item_class, const int64_t *nsteps,
                           const double *t0, const double *y0, const double *params, const double *counters);
/* Threads per block (32..256, multiple of 32) and resident blocks per SM
 * (0 = as many as fit).  Classes with lanes per orbit use 8 x
 * (32 / lanes) x (slot) bytes of shared memory per warp; a block size whose
 * warps need more than 48 KiB in all is rejected. */
int sodecl_batch_set_launch(sodecl_batch *b, int32_t block, int32_t blocks_per_sm);
/* Autotuner: times candidate lanes per orbit for the classes whose
 * lanes_per_orbit is automatic (rebuilding the program for each), then every
 * candidate launch shape, on the current items (each trial advances them),
 * and keeps the fastest. */
int sodecl_batch_tune(sodecl_batch *b, int32_t *block, int32_t *blocks_per_sm, double *best_ms);
/* Lanes per orbit each class runs with (one entry per class). */
int sodecl_batch_class_lanes(const sodecl_batch *b, int32_t *lanes);
/* One persistent launch over every item from its current state; use_graph:
 * replay a captured CUDA graph (captured on first use). */
int sodecl_batch_run(sodecl_batch *b, int32_t use_graph);
/* Final states in the caller's orbit order and packing; any pointer may be NULL. */
int sodecl_batch_results(sodecl_batch *b, double *t, double *y, double *counters, int64_t *newton_passes,
                         int32_t *flags);
int sodecl_batch_last_ms(const sodecl_batch *b, double *ms);
int sodecl_batch_kernel_info(sodecl_batch *b, int *regs, int *local_bytes);
size_t sodecl_batch_last_error(const sodecl_batch *b, char *buf, size_t n);

/* Allocation-free launch of a compiled batch.  No counterpart in the
 * reference.  For callers that cannot let a library call cudaMalloc -- a
 * custom operator inside a framework whose allocator owns all device memory,
 * or a service that allocates its working set once at start-up -- because an
 * allocation (or free) in their launch path synchronises the device and
 * fragments memory they manage.  The caller passes every input and output as
 * device memory it owns: orbits grouped by class (class 0's first, then
 * class 1's, ...; counts in the host array class_count, one entry per class),
 * states and parameters packed in that order with each class's widths.  The
 * kernel's only scratch, one work-queue head per class, is a 256-byte
 * file-scope device array inside the library (at most 32 classes; more is
 * rejected): every GPU that loads the library holds it until exit, every call
 * on a device shares it, each call clears it on `stream` before its launch,
 * and calls that overlap on the GPU race on it.  The first call on a device
 * loads the batch program there and looks up the array's address; make that
 * first call before any stream capture.  The cached address and the loaded
 * program belong to the device's context as it was at that first call: after
 * a cudaDeviceReset in the same process, this entry point must not be used
 * again.  Returns after queuing the launch on `stream`; the noise stream of
 * an orbit is keyed by its position.
 *
 * Scheduling: within a class, orbits are taken in the caller's order (the
 * regular entry point sorts each class by decreasing step count so that the
 * longest orbits start first; this one does not sort, because sorting would
 * need scratch for the permutation).  Put long orbits first for the same
 * load balance.
 *
 * Inputs are not validated on the host beyond null checks and the kind of
 * memory (as for sodecl_cuda_launch: memory the device cannot access is
 * refused): every pointer but class_count must be device memory the caller
 * owns, sized for the counts in class_count, whose contents the host never
 * reads; a step count of zero or less takes no step and leaves that
 * orbit's state unchanged. */
typedef struct sodecl_batch_io {
    double *t;                  /* device, [n] in/out */
    double *y;                  /* device, states, in/out */
    const double *params;       /* device, parameters */
    double *counters;           /* device, [n] in/out, or NULL when no class is stochastic */
    const int64_t *nsteps;      /* device, [n]; <= 0 takes no step */
    int64_t *newton_passes;     /* device, [n] out, or NULL */
    int32_t *flags;             /* device, [n] out, or NULL */
    const int64_t *class_count; /* host, one count per class */
} sodecl_batch_io;

int sodecl_batch_run_noalloc(sodecl_batch *b, const sodecl_batch_io *io, void *stream);
size_t sodecl_batch_program_source(const sodecl_batch *b, char *buf, size_t n);
void sodecl_batch_destroy(sodecl_batch *b);

/* ---- test and measurement helpers -------------------------------------- */

/* The Euler-Maruyama noise stream computed on the GPU by the same device
 * code the solver uses.  For each of n orbits (global ids gids[i], starting
 * draw counters counters[i]) and nsteps steps: Gaussian increments
 * normals[(i*nsteps + s)*nnoi + k] for step `dt_program` (the printed step),
 * and optionally the raw Threefry words and (0,1) doubles of every draw,
 * words/u01[((i*nsteps + s)*ncalls + c)*2 + {0,1}], ncalls = (nnoi+1)/2.
 * Host pointers. */
int sodecl_cuda_noise_stream(int device, const int64_t *gids, const double *counters, int64_t n, int32_t nnoi,
                             double dt_program, int64_t nsteps, double *normals, uint64_t *words, double *u01);

/* Compares the reciprocal quotient of SODECL_DIV_RECIPROCAL with IEEE
 * division, bit for bit, on `pairs` pseudo-random operand pairs (every
 * exponent, significands near 1 and 2, zeros, subnormals, Inf, NaN) drawn
 * from `seed`.  Writes the number of differing results and the first
 * differing pair. */
int sodecl_cuda_division_check(int device, int64_t pairs, uint64_t seed, int64_t *mismatches, double *first_a,
                               double *first_b);

/* The same for FP32 programs' reciprocal quotient (binary32, fast path for
 * |a|, |b| in [2^-60, 2^60)) against IEEE float division. */
int sodecl_cuda_division_check_f32(int device, int64_t pairs, uint64_t seed, int64_t *mismatches, float *first_a,
                                   float *first_b);

/* Issue-rate microbenchmark of the FP64 (precision 0) or FP32 (1) FMA pipe:
 * independent FMA chains on every SM, timed with CUDA events, the fastest
 * of seven launches after two warm-up launches.  Writes the FMA
 * instructions per second summed over all lanes (one FMA = 2 flops) and
 * that launch's time. */
int sodecl_cuda_fma_peak(int device, int32_t precision, double *fma_per_s, double *ms);

/* Throughput microbenchmark of the math library's sin in FP64 (precision 0)
 * or FP32 (1): eight independent sums of sin(x_k - y) per thread on every SM,
 * with arguments within a few units of zero, the coupling term of the
 * Kuramoto right-hand side.  Timed as sodecl_cuda_fma_peak; writes sines
 * per second and that launch's time.  It is the ceiling of a right-hand side
 * made of sine evaluations, as the FMA rate is of plain arithmetic.  No
 * counterpart in the reference (a measurement of this library's own). */
int sodecl_cuda_sin_peak(int device, int32_t precision, double *sin_per_s, double *ms);

#ifdef __cplusplus
}
#endif

#endif /* SODECL_CUDA_H */
