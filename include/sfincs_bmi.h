/*
 * C-ABI of libsfincs_gpu.so: the B200 SFINCS time-stepping core.
 *
 * The first block replaces the reference's BMI/XMI shared-library surface
 * one for one (source/src/sfincs_bmi.f90, built as sfincs.dll/libsfincs.so and
 * bound by xmipy or any iso_c_binding caller): same symbol names, argument
 * passing (by reference unless the Fortran declares `value`), return codes
 * (0 = success) and 1-based cell indices.  The remaining blocks are additions
 * with no counterpart in the reference.
 *
 * Threading: like the reference (module-level state), the BMI block drives
 * ONE global model per process; callers serialise calls.  The sfg_model_* and
 * sfg_ensemble_* handles are independent objects.
 */
#ifndef SFINCS_BMI_H
#define SFINCS_BMI_H

#include <stddef.h>

#if defined(__GNUC__)
#define SFG_API __attribute__((visibility("default")))
#else
#define SFG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- BMI string-length constants (sfincs_bmi.f90:41-52) ------------------ */
extern SFG_API int BMI_LENVARADDRESS;    /* 64   */
extern SFG_API int BMI_LENVARTYPE;       /* 64   */
extern SFG_API int BMI_LENGRIDTYPE;      /* 64   */
extern SFG_API int BMI_LENCOMPONENTNAME; /* 64   */
extern SFG_API int BMI_LENVERSION;       /* 256  */
extern SFG_API int BMI_LENERRMESSAGE;    /* 1024 */

/* ---- lifecycle ------------------------------------------------------------- */
/* sfincs_bmi.f90:56-63.  Reads ./sfincs.inp (current working directory), sets
 * use_qext, builds the device-resident model on the current CUDA device.
 * Returns 0, or non-zero with get_last_bmi_error() describing the failure
 * (the reference stops the process on bad input instead). */
SFG_API int initialize(void);
/* sfincs_bmi.f90:65-73: exactly one time step (if t < tstop). */
SFG_API int update(void);
/* sfincs_bmi.f90:75-85: step while t < t_target (the last step may overshoot). */
SFG_API int update_until(double t_target);
/* sfincs_bmi.f90:87-93: releases the model; returns 1 if the run stopped on
 * the minimum-time-step instability check (sfincs_lib.f90:634-648, 807-815). */
SFG_API int finalize(void);

/* ---- data exchange ---------------------------------------------------------- */
/* sfincs_bmi.f90:95-129.  Host pointers owned by the library, valid until
 * finalize().  Names: "z_xz","z_yz","zb","subgrid_z_zmin","qext" (float[np]),
 * "zs" (double[np]).  "zs" is refreshed from the device after every
 * update()/update_until() once its pointer has been taken; "qext" is copied to
 * the device before every update()/update_until() once its pointer has been
 * taken.  Unknown or unavailable names: *ptr = NULL, returns -1. */
SFG_API int get_value_ptr(const char* name, void** ptr);
/* sfincs_bmi.f90:131-157: shape[0] = np for the names above. */
SFG_API int get_var_shape(const char* name, int shape[6]);
/* sfincs_bmi.f90:159-185: "float", "double" or "integer" into type[BMI_LENVARTYPE]. */
SFG_API int get_var_type(const char* name, char* type);
/* sfincs_bmi.f90:187-207 */
SFG_API int get_var_rank(const char* name, int* rank);
/* sfincs_bmi.f90:209-235: only "qext" (switches the external source term). */
SFG_API int set_logical(const char* name, const int* value);

/* ---- time (sfincs_bmi.f90:237-275) -------------------------------------------- */
SFG_API int get_start_time(double* t);
SFG_API int get_end_time(double* t);
SFG_API int get_time_step(double* dt);
SFG_API int get_current_time(double* t);

/* ---- extras -------------------------------------------------------------------- */
/* sfincs_bmi.f90:277-284: re-derive zbuvmx (and the device bed level) after the
 * caller edited "zb" through its pointer. */
SFG_API int update_zbuv(void);
/* sfincs_bmi.f90:286-297: wave-enhanced roughness is not part of this core
 * (initialize() rejects inputs that enable it); returns 0 without effect. */
SFG_API int update_apparent_roughness(void);
/* sfincs_bmi.f90:299-316: 1-based active-cell index of point (x, y), 0 if outside. */
SFG_API int get_sfincs_cell_index(const double* x, const double* y, int* index);
/* sfincs_bmi.f90:318-349: n points, n passed by value. */
SFG_API int get_sfincs_cell_indices(const double* x, const double* y, int* index, int n);
/* sfincs_bmi.f90:351-373: area (m2) of 1-based cell index. */
SFG_API int get_sfincs_cell_area(const int* index, double* area);
/* sfincs_bmi.f90:378-387: last error message into msg[BMI_LENERRMESSAGE]. */
SFG_API int get_last_bmi_error(char* msg);

/* ---- additions (no counterpart in the reference) -------------------------------- */
/* initialize() for a model directory other than the working directory. */
SFG_API int initialize_config(const char* model_dir);
/* Copy-based access: "zs" (double[np]), "zsmax","qext" (float[np]),
 * "z_volume" (double[np], subgrid), "qx","qy","uvx","uvy" (float[np]: flux /
 * velocity of each cell's right (x) or upper (y) face, 0 where no face);
 * with their store switches on, "vmax","qmax","twet","tzsmax","cumprcp",
 * "cuminf" (float[np]: maximum velocity and flux, wet duration, time of the
 * maximum level, cumulative rain and infiltration).
 * bytes must equal the array size. */
SFG_API int get_var(const char* name, void* dst, size_t bytes);
SFG_API int set_var(const char* name, const void* src, size_t bytes);

/* ---- model handles: independent models (no global state) ------------------------- */
/* Create a device-resident model from <model_dir>/sfincs.inp.  bmi != 0 turns
 * the external source term (qext) on, as initialize() does.  NULL on error;
 * the message is then in err[errlen]. */
SFG_API void* sfg_model_create(const char* model_dir, int bmi, char* err, int errlen);
SFG_API void sfg_model_destroy(void* model);
/* finalize_output (sfincs_output.f90:260-296): the last max-output interval,
 * the run's scalars, the map / his files closed.  finalize() does this for the
 * BMI model; sfg_model_destroy does it when it was not called, without an
 * error report. */
SFG_API int sfg_model_finalize(void* model);
/* sfincs_update semantics: run while t < t_end, at most max_steps steps when
 * max_steps >= 0; steps are issued as CUDA graphs of `chunk` steps. */
SFG_API int sfg_model_run(void* model, double t_end, long long max_steps, int chunk);
/* Issue nsteps steps on the model's stream without waiting (timing helper). */
SFG_API int sfg_model_issue(void* model, int nsteps);
/* Kernel variant: 5 (default) and 4 are the TMA-staged tile kernels compiled
 * for 4 and 3 CTAs per SM, 2 and 3 the per-thread-load kernels.  All compute
 * bitwise identical states.  With autotune on, the next run() times one
 * chunk of real steps with each of 5, 4 and 2 and keeps the fastest. */
SFG_API int sfg_model_set_autotune(void* model, int on);
SFG_API int sfg_model_variant(void* model);
SFG_API int sfg_model_set_variant(void* model, int variant);
SFG_API int sfg_model_sync(void* model);
/* [t, dt, min_dt, nt, error, t0, t1, np, npuv, nkcuv2, ngbnd, subgrid,
 *  bflux_vol, rain_vol, src_vol, dtmax, dtmin, device_bytes, ntiles] */
SFG_API int sfg_model_scalars(void* model, double out[19]);
/* Same names as get_var, plus "kfuv" (float[2*np]: u then v face wet flags). */
SFG_API int sfg_model_get(void* model, const char* name, void* dst, size_t bytes);
SFG_API int sfg_model_set(void* model, const char* name, const void* src, size_t bytes);
/* Total water volume (m3, FP64) of the active cells; subgrid: sum of z_volume. */
SFG_API int sfg_model_volume(void* model, double* volume);
/* The same sum (bit for bit) for callers that must not allocate device memory
 * when they ask for it; no counterpart in the reference.  Its scratch (4096
 * FP64 partial sums and the total) is a fixed array inside the library, one
 * per device and shared by every model on it, so calls that overlap in time
 * race and must be serialised.  The first call on a device looks the array
 * up; make it before any stream capture begins.  Synchronises the model's
 * stream.  Returns 0, or 1 with the reason in get_last_bmi_error(). */
SFG_API int sfg_model_volume_noalloc(void* model, double* volume);
/* CUDA stream the model's kernels run on (cudaStream_t), for event timing. */
SFG_API void* sfg_model_stream(void* model);
/* Run nsteps steps with CUDA events between the individual launches (on the
 * model's stream) and return the mean duration in ms of the
 * [step+boundary, momentum, point sources, continuity] launches in ms_out[4];
 * launches_per_step receives how many kernels one step launches. */
SFG_API int sfg_model_kernel_times(void* model, int nsteps, double ms_out[4], int* launches_per_step);

/* ---- ensembles: many uneven models advanced by the same launches -------------------- */
SFG_API void* sfg_ensemble_create(const char* const* model_dirs, int n, int bmi, char* err, int errlen);
SFG_API void sfg_ensemble_destroy(void* ens);
/* Run every member to its own t_end[i] (per-member dt); steps issued in CUDA
 * graphs of `chunk` steps, host checks completion once per chunk. */
SFG_API int sfg_ensemble_run(void* ens, const double* t_end, long long max_steps, int chunk);
SFG_API int sfg_ensemble_issue(void* ens, int nsteps);
SFG_API int sfg_ensemble_set_autotune(void* ens, int on);
SFG_API int sfg_ensemble_variant(void* ens);
SFG_API int sfg_ensemble_set_variant(void* ens, int variant);
SFG_API int sfg_ensemble_sync(void* ens);
SFG_API int sfg_ensemble_scalars(void* ens, int member, double out[19]);
SFG_API int sfg_ensemble_get(void* ens, int member, const char* name, void* dst, size_t bytes);
SFG_API void* sfg_ensemble_stream(void* ens);
SFG_API int sfg_ensemble_kernel_times(void* ens, int nsteps, double ms_out[4], int* launches_per_step);

/* ---- serving pool: continuous batching of independent requests ------------------------ */
/* A pool of at most max_slots resident models whose device memory together
 * stays within hbm_budget_bytes.  Resident models advance together in the same
 * launches (per-model dt); models join and leave between chunks of steps. */
SFG_API void* sfg_pool_create(int max_slots, double hbm_budget_bytes, char* err, int errlen);
SFG_API void sfg_pool_destroy(void* pool);
/* Host-only preparation of a model (reads the inputs, builds the layout); no
 * device work, callable from any host thread while the pool is stepping. */
SFG_API void* sfg_prepare(const char* model_dir, int bmi, char* err, int errlen);
/* Exact device bytes the prepared model needs once admitted. */
SFG_API double sfg_prepared_bytes(void* prepared);
SFG_API double sfg_prepared_cells(void* prepared);
SFG_API void sfg_prepared_destroy(void* prepared);
/* Admit a prepared model to run until t_end (negative: the model's own tstop):
 * returns its slot (the pool then
 * owns the prepared model), -1 if no slot is free or the budget would be
 * exceeded (the prepared model stays the caller's), -2 on error. */
SFG_API int sfg_pool_admit(void* pool, void* prepared, double t_end);
/* Advance every running model by up to nsteps steps (CUDA graph chunks) and
 * return how many are still running (-2 on error). */
SFG_API int sfg_pool_advance(void* pool, int nsteps);
/* Slots whose model has finished (reached t_end or stopped), up to cap. */
SFG_API int sfg_pool_finished(void* pool, int* slots, int cap);
SFG_API int sfg_pool_scalars(void* pool, int slot, double out[19]);
/* "zs","z_volume" (double[np]); "zsmax","qx","qy","uvx","uvy" (float[np]). */
SFG_API int sfg_pool_get(void* pool, int slot, const char* name, void* dst, size_t bytes);
/* Free the slot and its device memory. */
SFG_API int sfg_pool_release(void* pool, int slot);
SFG_API double sfg_pool_used_bytes(void* pool);
SFG_API int sfg_pool_resident(void* pool);
SFG_API void* sfg_pool_stream(void* pool);

/* ---- diagnostics: host-side layout of a model, no device work -------------------------- */
/* Loads <model_dir> on the host only and copies one layout array (compact
 * reference cell order) into dst: "counts" (double[10]: np, npuv, ngbnd,
 * nkcuv2, nlevels, nalloc, dtmax, dtmin, t0, t1), "flags" (double[np]), "zs" and
 * "zvol" (initial state, double[np]), "zbmx","gn2" (double[2*np]: u then v
 * face of each cell), "gb_cell" (double[ngbnd], compact index), "kb_cell",
 * "kb_dir","kb_sign","kb_fac" (double[nkcuv2], water-level boundary faces in
 * reference order).  Returns 0 or -1. */
SFG_API int sfg_layout_get(const char* model_dir, int bmi, const char* name, double* dst, size_t n);

#ifdef __cplusplus
}
#endif

#endif /* SFINCS_BMI_H */
