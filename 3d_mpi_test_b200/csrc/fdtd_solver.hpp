// Host side of the B200 time-marching path: one device-resident domain per
// Solver, built from the reference's setup files.
#pragma once

#include <array>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "fdtd_input.hpp"

namespace fdtd {

struct SolverError {
    int code;
    std::string msg;
};

class SolverImplBase;
class EnsembleImplBase;

// Receiver post-processing on a device (fdtd_spectra.cu): the reference's
// zero-padded, 1/2^m-scaled forward FFT of each trace [nrec][nt], as the
// complex spectra [nrec][2^m], as magnitudes of bins [k0, k0 + nk), or as
// third-octave-style band levels 10 log10(sum |X_k|^2) [nrec][nband].
void fft_forward(int device, const double* traces, int nrec, int nt, int m, double* re, double* im);
void spectrum_bins(int device, const double* traces, int nrec, int nt, int m, long k0, long nk, double* mag);
void band_levels(int device, const double* traces, int nrec, int nt, int m, double dt, int nband, const double* fc,
                 double* levels);

class Solver {
   public:
    // precision: 0 FP64, 1 FP32. Throws SolverError.
    Solver(const std::string& case_dir, int precision, int device);
    ~Solver();
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    const ReferenceInput& input() const;
    std::array<int, 12> dims() const;
    int precision() const { return precision_; }

    // receivers at reference coordinates; returns whole-domain indices (3 per receiver)
    std::vector<int> set_receivers(const std::vector<double>& xyz);
    int n_receivers() const;

    // back to t = 0; horizon = planned steps (<= 0: input.txt's time_domain)
    void reset(int horizon = 0);
    // time loop; rec_out: [n][nrec] host FP64 or nullptr. Returns steps taken.
    int run(int nsteps, double* rec_out);
    int advance(int nsteps, double* rec_out);
    void step_pressure();
    void step_velocity();

    void get_field(int medium, int comp, double* out);
    void set_field(int medium, int comp, const double* in);
    void get_psi(double* out);
    // impedance-ground TDBC state [i][j][6], FP64 (tdbc_ground.dat)
    void get_ground_psi(double* out);
    int get_slab(int s, int comp, double* out, int* dims);
    size_t state_elems() const;
    void copy_state(int dir, void* host);
    void save_restart(const std::string& path);
    void write_contour(const std::string& path, int format);
    void load_restart(const std::string& path, bool reference_semantics);
    long long launch_count() const;
    void set_tiling(int rows_per_block, int planes_per_block, int threads_per_block, int vector_width,
                    int ring_stages);
    std::array<int, 5> autotune(int nsteps);
    double last_device_ms() const;
    // receiver samples of steps [first_step, first_step + nsteps) already taken
    void get_receivers(int first_step, int nsteps, double* out);
    // polls of a staged-copy wait before the fused pass reports a timeout
    // (0: at once; < 0: the default)
    void set_wait_limit(long long polls);
    // tiled FB_p_v kernel: shape of the full (kind 0) or lean (1) tiles --
    // rows, column vectors and planes per tile, ring stages; selects it
    void set_tile_shape(int kind, int rows, int vectors, int planes, int stages);
    // {per kind: rows, vectors, planes, stages, threads, tiles} x 2, tiled kernel on
    std::array<int, 19> tile_shape() const;
    // block timeline of the tiled kernels: per step slot (64) and tile kind
    // (10) earliest start, latest end, summed durations (ns) and blocks
    void set_block_trace(bool on);
    void get_block_trace(unsigned long long* out);

   private:
    friend class Ensemble;
    int precision_;
    std::unique_ptr<SolverImplBase> impl_;
};

// Independent solvers of one precision on one device stepped together by
// batched launches of the marching kernel (fused FB_p_v members without the
// moving frame). The solvers stay owned by the caller and keep their own
// setup, read-out and receiver buffers; they must outlive the ensemble.
class Ensemble {
   public:
    explicit Ensemble(const std::vector<Solver*>& members);
    ~Ensemble();
    Ensemble(const Ensemble&) = delete;
    Ensemble& operator=(const Ensemble&) = delete;
    // lock-step steps of every member; returns the steps taken (the nearest
    // member horizon bounds it)
    int advance(int nsteps);
    // one tile rule for all members: returns {rows per block, planes per block}
    std::array<int, 2> autotune(int nsteps);
    double last_device_ms() const;
    long long launch_count() const;
    // {launch groups, blocks per step}
    std::array<long long, 2> shape() const;
    // 0: one batched launch per group per step; 1 (default): every member's
    // own marching launch, members spread over several streams
    void set_mode(int mode);

   private:
    std::unique_ptr<EnsembleImplBase> impl_;
};

}  // namespace fdtd
