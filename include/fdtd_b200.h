/*
 * fdtd_b200.h -- C ABI of the B200 (sm_100a) time-marching path of the
 * outdoor-sound FDTD solver whose reference is azhang22/3D_MPI_TEST.
 *
 * One handle = one device-resident domain (air + optional porous ground)
 * built from a reference case directory (input.txt + coordi_*.dat). The
 * library owns all device memory; host buffers are caller-owned. Every
 * function returns an int status (FDTD_OK or a negative FDTD_ERR_*);
 * fdtd_last_error() returns the message of the calling thread's last
 * failure. A handle is not thread-safe: use one handle per host thread.
 *
 * Reference interfaces replaced (file:line in the reference repository):
 *   fdtd_create        airpore::airpore (airpore.cpp:17-316) +
 *                      airpore::SetInitialCond (airpore.cpp:936-964) +
 *                      air::air / porous::porous constructors
 *   fdtd_set_receivers calculation_2D::get_position (calculation_2D.cpp:317-352)
 *                      with the out-of-domain rule of airpore.cpp:454-457
 *   fdtd_run           airpore::get_output time loop (airpore.cpp:539-624):
 *                      SetMovingFrame + per step get_pressure, Cal_pressure,
 *                      Cal_velocity, UpdateInitialCond
 *   fdtd_advance       the same loop, continued from the current state
 *   fdtd_step_pressure airpore::Cal_pressure (airpore.cpp:366-398)
 *   fdtd_step_velocity airpore::Cal_velocity + UpdateInitialCond
 *                      (airpore.cpp:324-364, 648-662)
 *   fdtd_get_field     read-out of calculation_2D::p_n/u_n/v_n/w_n
 *                      (calculation_2D.h:33-34) in the reference [i][j][k] order
 *   fdtd_set_field     write of the same arrays (restart input,
 *                      calculation_2D.cpp:522-545)
 *   fdtd_get_psi       calculation_2D::Psi (TDBC state, calculation_2D.h:71)
 *   fdtd_get_ground_psi no counterpart: the state of the impedance-ground
 *                      TDBC (optional tdbc_ground.dat), an extension that
 *                      runs the east face's recursion (calculation_2D.cpp:
 *                      986-1017) on the ground face with fitted poles
 *   fdtd_get_slab      air::Qux1..Qpz2 PML integrals (air.h:40-42)
 *   fdtd_get_receivers the receiver series airpore::get_output collects
 *                      through get_pressure (airpore.cpp:566-580)
 *   fdtd_ensemble_*    no counterpart: the reference runs one case per MPI
 *                      job; an ensemble steps many handles' get_output loops
 *                      together
 */
#ifndef FDTD_B200_H
#define FDTD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDTD_OK 0
#define FDTD_ERR_INPUT (-1)       /* unreadable or malformed case files */
#define FDTD_ERR_UNSUPPORTED (-2) /* a configuration the reference itself cannot run */
#define FDTD_ERR_CUDA (-3)        /* CUDA runtime failure or no sm_100 device */
#define FDTD_ERR_NONFINITE (-4)   /* a pressure value became Inf/NaN */
#define FDTD_ERR_ARG (-5)         /* bad argument (null pointer, range) */
#define FDTD_ERR_STATE (-6)       /* time loop finished; call fdtd_reset */
#define FDTD_ERR_TIMEOUT (-7)     /* a staged plane copy did not land within the wait limit */

#define FDTD_F64 0
#define FDTD_F32 1

typedef struct fdtd_solver fdtd_solver;

/* dims[0..11]: air I J K, has_pore, pore I J K, unified NG, time_domain,
 * precision, scheme (0 FB_p_v, 1 FB_v_p), steps taken so far */
#define FDTD_NDIMS 12

int fdtd_create(const char *case_dir, int precision, int device, fdtd_solver **out);
int fdtd_destroy(fdtd_solver *h);
int fdtd_dims(const fdtd_solver *h, int *dims);
const char *fdtd_last_error(void);

/* Receivers at reference coordinates (X, Y, Z triples); idx_out (3n ints,
 * may be NULL) receives the whole-domain node indices. n <= 64. */
int fdtd_set_receivers(fdtd_solver *h, int n, const double *xyz, int *idx_out);

/* Back to the initial condition at t = 0, frame 0. horizon = the planned
 * number of steps (the reference's time_domain, which sets the last frame's
 * length and the receiver buffer); <= 0 keeps input.txt's value. */
int fdtd_reset(fdtd_solver *h, int horizon);

/* Reset, then run the reference time loop for nsteps steps (nsteps takes the
 * place of input.txt's time_domain). rec_out: host [nsteps][n_receivers]
 * FP64 pressure sampled before each step, or NULL. */
int fdtd_run(fdtd_solver *h, int nsteps, double *rec_out);

/* Continue the time loop by nsteps (frame schedule from input.txt's
 * time_domain); rec_out as above for the new steps, or NULL. */
int fdtd_advance(fdtd_solver *h, int nsteps, double *rec_out);

/* One half step each, for per-half-step parity: pressure then velocity
 * (FB_p_v). fdtd_step_velocity also swaps the time levels. */
int fdtd_step_pressure(fdtd_solver *h);
int fdtd_step_velocity(fdtd_solver *h);

/* medium 0 air, 1 porous ground; comp 0 p, 1 u, 2 v, 3 w. Host FP64 array
 * in [i][j][k] order (k fastest) of that medium's grid. */
int fdtd_get_field(fdtd_solver *h, int medium, int comp, double *out);
int fdtd_set_field(fdtd_solver *h, int medium, int comp, const double *in);

/* TDBC state [i][k][6] of the air grid (FP64). */
int fdtd_get_psi(fdtd_solver *h, double *out);

/* Impedance-ground TDBC state [i][j][6] (FP64) of a case with
 * tdbc_ground.dat; FDTD_ERR_UNSUPPORTED without one. Extension: the
 * reference's TDBC state exists for the east face only
 * (calculation_2D.h:71). */
int fdtd_get_ground_psi(fdtd_solver *h, double *out);

/* PML integral slab s (0 x1, 1 x2, 2 y1, 3 y2, 4 z1, 5 z2), comp 0 u 1 v 2 w
 * 3 p, in the reference slab shape [d0][d1][d2]. dims receives the shape;
 * returns 1 if the slab exists, 0 if not. out may be NULL. */
int fdtd_get_slab(fdtd_solver *h, int s, int comp, double *out, int *dims);

/* Whole device state in the native layout ([g][i][j] with each j row padded
 * to a multiple of 16 bytes, precision of the handle): 4 fields u v w p,
 * each fdtd_state_elems() elements. dir 0:
 * device -> host, 1: host -> device. Used for end-to-end timing with host
 * buffers. */
size_t fdtd_state_elems(const fdtd_solver *h);
int fdtd_copy_state(fdtd_solver *h, int dir, void *host);

/* Tile shape of the single-pass FB_p_v row marching kernel (selecting it
 * in place of the tiled kernel below): rows_per_block
 * i-rows x all j columns x planes_per_block g-planes per thread block. A
 * thread owns vector_width consecutive columns (0: 16 bytes of columns, i.e.
 * 4 in FP32 and 2 in FP64; else 2 or 4 with vector_width * element size <=
 * 16); a "thread row" is NJP / vector_width threads and threads_per_block
 * is rounded down to whole thread rows (at least 1, at most 256 threads and
 * rows_per_block + 1 thread rows). ring_stages: planes of the shared-memory
 * staging ring (0: the minimum, 3, or 4 with wind; each further stage keeps
 * one more plane in flight; at most 12). Takes effect for the next step.
 * Returns FDTD_ERR_ARG for a bad vector width or stage count and
 * FDTD_ERR_UNSUPPORTED when the tile does not fit shared memory or one
 * thread row exceeds 256 threads. */
int fdtd_set_tiling(fdtd_solver *h, int rows_per_block, int planes_per_block, int threads_per_block,
                    int vector_width, int ring_stages);

/* The tiled FB_p_v kernel (the default for FB_p_v): each thread block
 * marches one tile of rows x 16-byte column vectors x planes; tiles follow
 * the PML layers and their storage, so "full" tiles (kind 0: faces, PML
 * edges and corners, storage-only PML rows, TDBC, inclusions), "lean" tiles
 * (kind 1: interior air or porous ground) and single-layer tiles (kind 2:
 * inside one x, y or z PML layer; three launches, one per axis) run as up
 * to five launches per step. fdtd_set_tile_shape sets the largest tile of
 * a kind (rows >= 2, vectors >= 2, planes >= 1, ring_stages 3..12 planes
 * of the TMA staging ring; at most 384 threads = (rows + 1) x (vectors + 1))
 * and selects the tiled kernel again after fdtd_set_tiling; FDTD_ERR_ARG
 * for a bad shape, FDTD_ERR_UNSUPPORTED when it does not fit the device.
 * fdtd_get_tile_shape: out[19] = per kind (full, lean, single-layer) rows,
 * vectors, planes, stages, threads per block, tiles per step; out[18] = 1
 * when the tiled kernel is active. No counterpart in the reference (its
 * loops sweep the whole domain per half step, air.cpp:1476-2322). */
int fdtd_set_tile_shape(fdtd_solver *h, int kind, int rows, int vectors, int planes, int ring_stages);
int fdtd_get_tile_shape(const fdtd_solver *h, int *out);

/* Block timeline of the tiled kernel (a profiling aid; off by default).
 * With it on, every block of every tile kind records its span with the
 * GPU's global timer; each fdtd_advance / get_output call clears the record
 * first. fdtd_get_block_trace: out[64 * 10 * 4] = per step slot (step % 64)
 * and tile kind (0 full, 1 lean, 2 + LM the PML / face kind of layer set LM,
 * bit 0 x, bit 1 y, bit 2 z): earliest block start, latest block end (ns of
 * the global timer; start ~0 when the kind did not run), summed block
 * durations (ns) and blocks; a block's own duration is read on one SM,
 * while the earliest start and latest end compare readings of different
 * SMs. FDTD_ERR_ARG when the trace was never enabled.
 * No counterpart in the reference. */
int fdtd_set_block_trace(fdtd_solver *h, int on);
int fdtd_get_block_trace(fdtd_solver *h, unsigned long long *out);

/* Times each candidate tile on this handle's domain (nsteps FB steps each,
 * CUDA events), keeps the fastest and returns it in best[5] (rows, planes,
 * threads, vector width, ring stages); the state is reset to t = 0
 * afterwards. With the tiled kernel active it tunes the lean and then the
 * full tile shape (read them with fdtd_get_tile_shape) and best[] describes
 * the full tiles; after fdtd_set_tiling it tunes the row marching kernel. */
int fdtd_autotune(fdtd_solver *h, int nsteps, int *best);

/* Kernel launches issued since creation (both passes, graphs included). */
long long fdtd_launch_count(const fdtd_solver *h);

/* CUDA events around the last fdtd_advance's device work: milliseconds. */
int fdtd_last_device_ms(const fdtd_solver *h, double *ms);

/* Receiver samples of steps [first_step, first_step + nsteps) already
 * taken since the last reset (fdtd_advance, fdtd_ensemble_advance), as
 * out [nsteps][n_receivers] FP64. */
int fdtd_get_receivers(fdtd_solver *h, int first_step, int nsteps, double *out);

/* Polls a staged-copy wait of the marching kernel makes before the kernel
 * gives up on the plane, records the failure and finishes without hanging
 * (the step then returns FDTD_ERR_TIMEOUT; the state is not meaningful and
 * the handle needs fdtd_reset). 0 gives up at the first wait, which lets a
 * caller exercise the error path; < 0 restores the default (2^22 polls). */
int fdtd_set_wait_limit(fdtd_solver *h, long long polls);

/* Ensembles: independent handles of one precision on one device stepped
 * together, the time loop captured in a CUDA graph. By default (mode 1,
 * fdtd_ensemble_set_mode) each step launches every member's marching
 * kernel, the members spread over up to 16 streams. In mode 0 each step is
 * one launch of the batched marching kernel per group of members (same
 * kernel form and block size class) over a work list of (member, row
 * block, plane chunk), heaviest blocks first, the groups as parallel
 * chains.
 * Members must use the fused FB_p_v pass (FDTD_ERR_UNSUPPORTED otherwise)
 * and no moving frame; they keep their receivers, horizon and read-out, and
 * must outlive the ensemble. fdtd_ensemble_advance takes min(nsteps, the
 * steps left to the nearest member horizon) steps of every member and
 * stores that count in *taken (FDTD_ERR_STATE if a member has none left).
 * fdtd_ensemble_autotune times one tile rule for all members, nsteps
 * steps of the whole ensemble each, keeps the fastest and resets every
 * member to t = 0 with its horizon kept. Mode 0: rows per block x planes
 * per block of the batched marching kernel, in best[2]. Mode 1 with tiled
 * members: one set of tile shapes (full, lean, PML / face) from a few
 * candidates; best[2] = the lean tiles' rows and planes.
 * fdtd_ensemble_info: info[0] launches so far, info[1] groups (launches per
 * step), info[2] thread blocks per step. */
typedef struct fdtd_ensemble fdtd_ensemble;
int fdtd_ensemble_create(fdtd_solver *const *members, int n, fdtd_ensemble **out);
int fdtd_ensemble_destroy(fdtd_ensemble *e);
int fdtd_ensemble_advance(fdtd_ensemble *e, int nsteps, int *taken);
int fdtd_ensemble_autotune(fdtd_ensemble *e, int nsteps, int *best);
int fdtd_ensemble_info(const fdtd_ensemble *e, long long *info);
int fdtd_ensemble_last_device_ms(const fdtd_ensemble *e, double *ms);
/* mode 0: one batched launch per group per step, members' parameters read
 * from a table in global memory; 1 (default): every member's own marching
 * launch (parameters in the constant bank), the members spread over up to
 * 16 streams in the captured step graph. FDTD_ERR_ARG for other values. */
int fdtd_ensemble_set_mode(fdtd_ensemble *e, int mode);

/* Pressure contour of the current state (airpore::get_data_contour,
 * airpore.cpp:1014-1056; calculation_2D::mpi_send_data and operator<<,
 * calculation_2D.cpp:1030-1190) to `path` instead of the reference's
 * hard-coded cluster path: every 4th node along each axis plus the last,
 * Y of the current moving frame, the porous ground as a second zone.
 * format 0: the reference's Tecplot ASCII POINT file, byte for byte;
 * 1: binary -- "FDTDCNT1", int32 zones, per zone int32 I J K then float64
 * X[I], Y[J], Z[K], P[K][J][I]. */
int fdtd_write_contour(fdtd_solver *h, const char *path, int format);

/* Restart files (airpore::Save_restart / Read_restart, airpore.cpp:664-879;
 * calculation_2D::save/input_restart_cal, calculation_2D.cpp:497-545;
 * air::save/input_restart_air, air.cpp:1305-1474). fdtd_save_restart writes
 * the current state in the reference's single-rank text layout (header
 * "size rank index", then air fields, wind and PML integrals, porous fields)
 * followed by one block the reference does not write -- the moving-frame
 * counters and the TDBC state Psi -- so the restart is exact for those too;
 * the reference's reader ignores it. fdtd_load_restart reads such a file,
 * or a file written by the reference itself (no extra block: Psi starts at
 * zero and the run continues in frame 0, as the reference's restart does),
 * into a handle created for the same case; the index must lie below the
 * horizon of the last fdtd_reset. Values carry 11 significant digits.
 * reference_semantics = 1 continues exactly as the reference does after its
 * Read_restart: its frame loop restarts frame 0 with air::SetQMove(0), which
 * zeroes all PML integrals (air.cpp:2453-2517), and it has no TDBC state in
 * the file -- so those start from zero (no moving frame). 0 keeps every
 * value the file holds (an exact restart for files of this library). */
int fdtd_save_restart(fdtd_solver *h, const char *path);
int fdtd_load_restart(fdtd_solver *h, const char *path, int reference_semantics);

/* Receiver post-processing (replaces airpore::get_FFT_y1, airpore.cpp:966-1011,
 * with FFT / FFT_output, FFT.cpp:15-120). traces: host [nrec][nt] pressure
 * histories (fdtd_run output); each is zero-padded (or cut) to 2^fft_m
 * points and transformed on `device` by the reference's radix-2 FFT,
 * forward and scaled by 1/2^fft_m, with the reference's twiddle sequence
 * and rounding -- bit for bit the reference's result. fdtd_fft returns the
 * complex spectra re, im [nrec][2^fft_m]. 1 <= fft_m <= 24. */
int fdtd_fft(int device, const double *traces, int nrec, int nt, int fft_m, double *re, double *im);

/* Magnitudes |X_k| of the same transform for bins k = k0 .. k0+nk-1
 * (FFT_output prints k = 0 .. 2^(fft_m-1) at frequency k / (dt 2^fft_m));
 * mag [nrec][nk]. */
int fdtd_spectrum(int device, const double *traces, int nrec, int nt, int fft_m, long long k0, long long nk,
                  double *mag);

/* Band levels (extension, no counterpart in the reference): for each trace
 * and each band centre fc[b] > 0, 10 log10 of the sum of |X_k|^2 over the
 * bins whose frequency k / (dt 2^fft_m) lies in [fc 2^(-1/6), fc 2^(1/6))
 * -- third-octave bands for base-2 centres 1000 * 2^(n/3); -inf for a band
 * without bins. levels_db [nrec][nband]. The difference of two runs' levels
 * (ground minus free field) is the excess attenuation per band. */
int fdtd_band_levels(int device, const double *traces, int nrec, int nt, int fft_m, double dt, int nband,
                     const double *fc, double *levels_db);

/* Allocation-free single FB_p_v step. No counterpart in the reference: it
 * serves callers that cannot allocate device memory (a host that owns all
 * device memory through its own pool, or code that must avoid the implicit
 * synchronisation of cudaMalloc/cudaFree). One forward-backward step of a
 * rigid-walled air box (no PML, wind, TDBC or porous ground), the same
 * kernels as the handle path, on caller-owned device buffers in the native
 * layout [k][i][j] (j fastest), FDTD_F64 or FDTD_F32 elements. X, Y, Z are
 * host coordinate arrays (NI, NJ, NK nodes); dx dy dz the input.txt
 * spacings; stream a cudaStream_t (NULL: legacy default stream). It
 * allocates nothing: its scratch is a fixed 128 KiB __device__ array
 * compiled into the library, so each axis is limited to 4096 nodes
 * (larger grids return FDTD_ERR_ARG). The first call on a device resolves
 * that array's device address (make it before any stream capture). All
 * calls share the array and reset it themselves; calls that overlap on the
 * GPU race and must be serialised by the caller. The four output buffers
 * must not overlap each other or any input buffer (FDTD_ERR_ARG otherwise:
 * the step cannot run in place). Synchronises the stream before returning;
 * FDTD_ERR_NONFINITE if the new pressure is not finite. */
int fdtd_fb_step_noalloc(int precision, int NI, int NJ, int NK, const double *X, const double *Y,
                         const double *Z, double dx, double dy, double dz, double dt, double gamma,
                         double P0, double c0, const void *u_in, const void *v_in, const void *w_in,
                         const void *p_in, void *u_out, void *v_out, void *w_out, void *p_out,
                         void *stream);

#ifdef __cplusplus
}
#endif
#endif
