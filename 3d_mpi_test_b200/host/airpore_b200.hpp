// C++ host classes over the C ABI (include/fdtd_b200.h) with the names and
// call shapes of the reference's airpore / calculation_2D / air / porous
// (airpore.h:24-68, calculation_2D.h:20-127, air.h:24-90, porous.h:12-30),
// so a reference driver (main.cpp: airpore(input) -> get_output ->
// get_FFT_y1) reads the same against the B200 library.
//
// What moves to the device: the per-node loops of cal_fp / cal_fuvw, the
// boundary updates, the PML integral updates and the nn -> n copy run as
// one fused FB_p_v step per time step on the GPU (or as the two half steps
// Cal_pressure / Cal_velocity). The member functions the reference calls
// between them (UpdateInitialCond, Update_PML_Qp / Qvw, UpdateBC_*) keep
// their names so the reference's call order still compiles, and do what the
// device step already did: nothing more. MPI set-up is a no-op: one
// device-resident domain replaces the rank decomposition.
//
// Errors: every failing call throws b200::Error (code = the FDTD_ERR_*
// value, what() = the library's message); the reference printed and went on.
#pragma once

#include <array>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "fdtd_b200.h"

namespace b200 {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Position (mygeneral.h): reference coordinates X (transverse), Y (range),
// Z (height)
struct Position {
    double x = 0, y = 0, z = 0;
};

enum Precision { FP64 = FDTD_F64, FP32 = FDTD_F32 };

class airpore;

// One medium's view of the device domain: the reference's calculation_2D
// (calculation_2D.h:20-127). Fields are read from and written to the
// device in the reference [i][j][k] order.
class calculation_2D {
   public:
    calculation_2D(fdtd_solver* h, int medium);
    virtual ~calculation_2D() = default;

    int get_whole_IMAX() const { return I_; }
    int get_whole_JMAX() const { return J_; }
    int get_whole_KMAX() const { return K_; }

    // p_n / u_n / v_n / w_n (calculation_2D.h:33-34) of this medium: comp
    // 'p', 'u', 'v' or 'w'
    std::vector<double> field(char comp) const;
    void set_field(char comp, const std::vector<double>& v);
    // calculation_2D::get_pressure (calculation_2D.cpp:387-403) on the
    // current p_n: the node's pressure, 0 outside the strict interior
    double get_pressure(int ii, int jj, int kk) const;

    // the device step already swapped the time levels (ping-pong): no copy
    void UpdateInitialCond(int /*N*/) {}

   protected:
    fdtd_solver* h_;
    int medium_, I_ = 0, J_ = 0, K_ = 0;
};

// air (air.h): the PML integrals live on the device and advance inside the
// step; they are read here in the reference slab shapes
class air : public calculation_2D {
   public:
    explicit air(fdtd_solver* h) : calculation_2D(h, 0) {}
    void Update_PML_Qp() {}
    void Update_PML_Qvw() {}
    // slab s (0 x1, 1 x2, 2 y1, 3 y2, 4 z1, 5 z2), comp 'u' 'v' 'w' 'p';
    // empty when the slab does not exist
    std::vector<double> pml_slab(int s, char comp, std::array<int, 3>* dims = nullptr) const;
    // TDBC state Psi[i][k][6] (calculation_2D.h:71), FP64
    std::vector<double> psi() const;
    // impedance-ground TDBC state Psi[i][j][6] (extension, tdbc_ground.dat)
    std::vector<double> ground_psi() const;
};

// porous (porous.h): the Zwikker-Kosten ground grid
class porous : public calculation_2D {
   public:
    explicit porous(fdtd_solver* h) : calculation_2D(h, 1) {}
};

// airpore (airpore.h:24-68): owns the device domain built from a case
// directory (input.txt + coordi_*.dat [+ coordi_pore*.dat, terrain.dat,
// logwind.dat, advection.dat, tdbc_ground.dat])
class airpore {
   public:
    explicit airpore(const std::string& case_dir, Precision precision = FP64, int device = 0);
    ~airpore();
    airpore(const airpore&) = delete;
    airpore& operator=(const airpore&) = delete;

    void MPI_Initialize() {}  // one device-resident domain: no decomposition
    // airpore::SetInitialCond (airpore.cpp:936-964): back to t = 0, frame 0;
    // horizon = the planned step count (0: input.txt's time_domain)
    void SetInitialCond(int horizon = 0);
    // half steps of the whole domain (airpore.cpp:324-398)
    void Cal_pressure();
    void Cal_velocity();
    void UpdateInitialCond(int /*MF_count*/) {}  // done by Cal_velocity's level swap

    // receivers at reference coordinates (get_position,
    // calculation_2D.cpp:317-352); returns the node indices
    std::vector<std::array<int, 3>> set_receivers(const std::vector<Position>& r);
    // the get_output time loop (airpore.cpp:539-624): nsteps steps from t = 0
    // (0: input.txt's time_domain); receivers() then holds p(t)
    void get_output(int nsteps = 0);
    // continue the loop by nsteps, appending to receivers()
    void advance(int nsteps);
    // [step][receiver] pressure sampled before each step, FP64
    const std::vector<double>& receivers() const { return rec_; }
    int n_receivers() const { return nrec_; }
    int steps_taken() const;

    // airpore::get_FFT_y1's spectra (airpore.cpp:966-1011) as band levels
    // (dB) of each receiver series, zero-padded to 2^fft_m points, for band
    // centres fc (third-octave bands [fc 2^-1/6, fc 2^1/6)); dt = the time
    // step; [receiver][band]
    std::vector<double> band_levels(int fft_m, double dt, const std::vector<double>& centres) const;

    // restart files in the reference's text format (airpore.cpp:664-879)
    void Save_restart(const std::string& path);
    void Read_restart(const std::string& path, bool reference_semantics = false);
    // contour output (airpore.cpp:1014-1056) to a path
    void get_data_contour(const std::string& path, bool binary = false);

    air* AirMedia = nullptr;
    porous* south_pore = nullptr;  // null without porous ground
    int time_domain() const { return dims_[8]; }
    fdtd_solver* handle() const { return h_; }

   private:
    fdtd_solver* h_ = nullptr;
    int device_ = 0;
    std::unique_ptr<air> air_;
    std::unique_ptr<porous> pore_;
    std::array<int, FDTD_NDIMS> dims_{};
    int nrec_ = 0;
    std::vector<double> rec_;
};

}  // namespace b200
