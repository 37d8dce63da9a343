/*
 * CPU oracle: plain-C restatement of the reference FDTD time-marching path
 * (azhang22/3D_MPI_TEST, single MPI rank). TEST INFRASTRUCTURE ONLY: it is
 * the checker the tests, smoke() and bench.py's cpu_baseline compare the
 * B200 kernels against; no product code path links or calls it.
 *
 * Parity of this restatement is pinned against the unmodified reference
 * compiled under oracle/_ref/ (ref_harness) on generated cases.
 */
#ifndef FDTD_ORACLE_H
#define FDTD_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc;

/* Parses <case_dir>/input.txt and the coordi_* files exactly like
 * airpore::airpore + airpore::SetInitialCond (airpore.cpp:17-316,936-964).
 * Returns NULL and fills err on failure. */
orc *orc_create(const char *case_dir, char *err, int errlen);
void orc_destroy(orc *o);

/* dims[0..9] = I J K has_pore pI pJ pK time_domain scheme n_slabs */
int orc_dims(const orc *o, int *dims);

/* Receiver positions (X,Y,Z triples) -> node indices, airpore.cpp:431-457. */
int orc_set_receivers(orc *o, int n, const double *xyz, int *idx_out);

/* Runs the airpore::get_output frame loop (airpore.cpp:539-624) for
 * nsteps steps (nsteps replaces time_domain); rec_out[nsteps*n] may be NULL. */
int orc_run(orc *o, int nsteps, double *rec_out);

/* medium 0 = air, 1 = porous ground; comp 0 p, 1 u, 2 v, 3 w; [i][j][k]. */
int orc_get_field(const orc *o, int medium, int comp, double *out);
int orc_set_field(orc *o, int medium, int comp, const double *in);
/* TDBC state [i][k][6] of the air grid. */
int orc_get_psi(const orc *o, double *out);
/* Impedance-ground TDBC state [i][j][6] (tdbc_ground.dat); -1 without one. */
int orc_get_ground_psi(const orc *o, double *out);
/* slab 0..5 = x1 x2 y1 y2 z1 z2; comp 0 u 1 v 2 w 3 p. dims[3] out.
 * Returns 1 if the slab exists, 0 if not. */
int orc_get_slab(const orc *o, int slab, int comp, double *out, int *dims);
/* Wind arrays Uav/Vav/Wav [i][j][k] (comp 0/1/2). */
int orc_get_wind(const orc *o, int comp, double *out);

/* In-place radix-2 FFT of 2^m points (FFT.cpp:15-83): dir 1 forward
 * (scaled by 1/2^m), -1 inverse. */
void orc_fft(int dir, int m, double *re, double *im);

#ifdef __cplusplus
}
#endif
#endif
