// Reference setup front end: input.txt + coordi_*.dat, parsed with the same
// positional rules as airpore::airpore (airpore.cpp:17-316) and
// calculation_2D::calculation_2D (calculation_2D.cpp:44-204).
#pragma once

#include <string>
#include <vector>

namespace fdtd {

// boundary_type (mygeneral.h:49)
enum BoundaryType { BT_RIGID = 0, BT_ABSORBING = 1, BT_POROUS = 2, BT_RADIATION = 3, BT_TDBC = 4 };
// scheme_list (mygeneral.h:48); only the forward-backward pair is implemented by the reference
enum Scheme { FB_P_V = 0, FB_V_P = 1, FB_VP = 2, LEAPTRAP = 3, ABM = 4, RK4 = 5, RK2 = 6 };

struct MovingFrameCfg {
    int JMAX = 0, lead_DJ = 2, trail_DJ = 2, Judge = 0;
    double ratio = 0.0;
};

struct AxisFile {
    int IMAX = 0, IMAX1 = 0, IMAX2 = 0, JMAX = 0, JMAX1 = 0, JMAX2 = 0, KMAX = 0, KMAX1 = 0, KMAX2 = 0, IJKMAX = 0;
    std::vector<double> X, Y, Z;  // whole axes as read (Y holds JMAX values)
};

struct ZKParams {  // PoreStruct / hillpore subset (airpore.cpp:249-295)
    double q = 1, porosity = 1, resistivity = 0, eff_density = 1, Kp = 1;
};

struct ReferenceInput {
    double gauss_width = 0;
    MovingFrameCfg mf;
    Scheme scheme = FB_P_V;
    BoundaryType north = BT_RIGID, south = BT_RIGID, east = BT_RIGID, west = BT_RIGID, front = BT_RIGID,
                 back = BT_RIGID;
    int case_no = 0;
    int pml_judge_x = 0, pml_judge_y = 0, pml_judge_z = 0;  // 0 none, 1 low side, 2 high side, 3 both
    int time_domain = 0, out_difft = 0, fft_m = 0;
    double frequency = 0;
    double velocity_coef = 0;
    int velocity_method = 0;
    double gamma = 1.4, P0 = 1e5, c0 = 340, Aav = 0;
    double pml_x_alpha = 0, pml_x_sigma = 0, pml_y_alpha = 0, pml_y_sigma = 0, pml_z_alpha = 0, pml_z_sigma = 0;
    int pml_y_time = 0;
    ZKParams pore;
    double Z_inf = 0, tau = 0;  // TDBC impedance scale and relaxation time (airpore.cpp:252-254)
    double source[3] = {0, 0, 0}, receiver[3] = {0, 0, 0};
    double dt = 0, dx = 0, dy = 0, dz = 0;
    double pdx = 0, pdy = 0, pdz = 0;
    int restart = 0, restart_out = 0;
    std::string restart_infile;
    int curve_judge = 0, curve_points = 0;
    double curve[12] = {0};
    ZKParams hill, canopy, trunk;
    double hill_box[6] = {0};
    AxisFile air, pore_axes;
    bool has_pore = false;
    // terrain-following grid (extension, optional terrain.dat: the count of Y
    // nodes, then the ground elevation at each); empty: flat ground
    std::vector<double> terrain;
    // log-law wind (extension, method 7): V = (velocity_coef / kappa) ln(z / z0),
    // optional logwind.dat holding kappa and z0
    double wind_kappa = 0.41, wind_z0 = 0.01;
    // velocity advection by the mean wind (extension, optional advection.dat:
    // "reference" forward differences as air.cpp:1476-1949, or "upwind"
    // backward differences)
    bool upwind_advection = false;
    // impedance ground (extension, optional tdbc_ground.dat: Zinf tau, six a,
    // six r): the rigid south face becomes a 6-pole TDBC with the east
    // face's recursion (calculation_2D.cpp:986-1017) and these poles
    bool ground_tdbc = false;
    double g_zinf = 0.0, g_tau = 0.0, g_a[6] = {0}, g_r[6] = {0};
};

// Returns "" on success, otherwise a one-line error.
std::string parse_reference_case(const std::string& case_dir, ReferenceInput& out);

}  // namespace fdtd
