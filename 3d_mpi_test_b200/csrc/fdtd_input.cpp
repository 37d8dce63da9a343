// Positional parser for the reference's input.txt and axis files.
//
// The reference reads input.txt with operator>> and skips comments with
// istream::ignore(100, '\n') (airpore.cpp:17-316); the same token/skip
// sequence is reproduced here so that any input the reference accepts
// yields the same values. Axis files: calculation_2D.cpp:44-204.
#include "fdtd_input.hpp"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace fdtd {
namespace {

struct Reader {
    std::string s;
    size_t pos = 0;
    bool fail = false;

    void ws() {
        while (pos < s.size() && std::isspace(static_cast<unsigned char>(s[pos]))) ++pos;
    }
    double d() {
        ws();
        const char* b = s.c_str() + pos;
        char* e = nullptr;
        double v = std::strtod(b, &e);
        if (e == b) { fail = true; return 0.0; }
        pos += static_cast<size_t>(e - b);
        return v;
    }
    int i() {
        ws();
        const char* b = s.c_str() + pos;
        char* e = nullptr;
        long v = std::strtol(b, &e, 10);
        if (e == b) { fail = true; return 0; }
        pos += static_cast<size_t>(e - b);
        return static_cast<int>(v);
    }
    std::string word() {
        ws();
        size_t b = pos;
        while (pos < s.size() && !std::isspace(static_cast<unsigned char>(s[pos]))) ++pos;
        return s.substr(b, pos - b);
    }
    // istream::ignore(100, '\n')
    void skip() {
        for (int c = 0; c < 100 && pos < s.size(); ++c)
            if (s[pos++] == '\n') break;
    }
};

bool slurp(const std::string& path, std::string& out) {
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

std::string read_axes(const std::string& dir, const std::string& prefix, AxisFile& ax) {
    std::string t;
    if (!slurp(dir + "/" + prefix + "1.dat", t)) return "cannot open " + dir + "/" + prefix + "1.dat";
    Reader r{t};
    ax.IMAX = r.i(); ax.IMAX1 = r.i(); ax.IMAX2 = r.i();
    ax.JMAX = r.i(); ax.JMAX1 = r.i(); ax.JMAX2 = r.i();
    ax.KMAX = r.i(); ax.KMAX1 = r.i(); ax.KMAX2 = r.i();
    ax.IJKMAX = r.i();
    if (r.fail || ax.IMAX <= 0 || ax.JMAX <= 0 || ax.KMAX <= 0) return "malformed header in " + prefix + "1.dat";
    ax.X.resize(ax.IMAX);
    for (auto& v : ax.X) v = r.d();
    if (r.fail) return "too few X coordinates in " + prefix + "1.dat";
    if (!slurp(dir + "/" + prefix + "2.dat", t)) return "cannot open " + dir + "/" + prefix + "2.dat";
    Reader r2{t};
    ax.Y.resize(ax.JMAX);
    for (auto& v : ax.Y) v = r2.d();
    if (r2.fail) return "too few Y coordinates in " + prefix + "2.dat";
    if (!slurp(dir + "/" + prefix + "3.dat", t)) return "cannot open " + dir + "/" + prefix + "3.dat";
    Reader r3{t};
    ax.Z.resize(ax.KMAX);
    for (auto& v : ax.Z) v = r3.d();
    if (r3.fail) return "too few Z coordinates in " + prefix + "3.dat";
    return "";
}

void set_zk(ZKParams& p, double Aav, double gamma, double P0) {
    p.eff_density = p.q * p.q / p.porosity / Aav;
    p.Kp = 1.0 / gamma / P0;
}

}  // namespace

std::string parse_reference_case(const std::string& dir, ReferenceInput& in) {
    std::string txt;
    if (!slurp(dir + "/input.txt", txt)) return "cannot open " + dir + "/input.txt";
    Reader r{txt};
    in.gauss_width = r.d(); r.skip();
    in.mf.JMAX = r.i(); in.mf.lead_DJ = r.i(); in.mf.trail_DJ = r.i(); in.mf.Judge = r.i(); in.mf.ratio = r.d();
    r.skip();
    const int st = r.i();
    r.skip();
    static const Scheme kSchemes[8] = {FB_P_V, FB_V_P, FB_P_V, FB_VP, LEAPTRAP, RK4, RK2, ABM};
    in.scheme = (st >= 1 && st <= 7) ? kSchemes[st] : FB_P_V;
    int bch[6];
    for (int& b : bch) b = r.i();
    r.skip(); r.skip();
    // Face order of line 4: North South East West Front Back (airpore.cpp:52-159).
    BoundaryType* direct[6] = {&in.north, &in.south, &in.east, &in.west, &in.front, &in.back};
    BoundaryType* radiation[6] = {&in.north, &in.south, &in.west, &in.east, &in.back, &in.front};
    int num_pml[3] = {0, 0, 0};
    for (int f = 0; f < 6; ++f) {
        switch (bch[f]) {
            case 1: *direct[f] = BT_RIGID; break;
            case 2: *direct[f] = BT_ABSORBING; num_pml[f / 2] += (f % 2 == 0) ? 1 : 10; break;
            case 3: *direct[f] = BT_POROUS; break;
            case 4: *radiation[f] = BT_RADIATION; break;
            case 5: if (f == 2) in.east = BT_TDBC; break;
            default: break;
        }
    }
    in.case_no = (in.north == BT_ABSORBING || in.north == BT_RIGID) ? 1
                 : (in.north == BT_POROUS)                          ? 2
                 : (in.north == BT_RADIATION)                       ? 3
                                                                     : 0;
    in.time_domain = r.i(); in.out_difft = r.i(); in.fft_m = r.i(); in.frequency = r.d(); r.skip();
    in.velocity_coef = r.d(); in.velocity_method = r.i(); r.skip();
    in.gamma = r.d(); in.P0 = r.d(); in.c0 = r.d(); r.skip();
    in.Aav = std::pow(in.c0, 2) / in.gamma / in.P0;
    in.pml_x_alpha = r.d(); in.pml_x_sigma = r.d(); r.skip();
    in.pml_y_alpha = r.d(); in.pml_y_sigma = r.d(); in.pml_y_time = r.i(); r.skip();
    in.pml_z_alpha = r.d(); in.pml_z_sigma = r.d(); r.skip();
    // num_PML slots: [0] z (North +1, South +10), [1] y (East +1, West +10), [2] x (Front +1, Back +10)
    auto judge = [](int n) { return n == 1 ? 2 : n == 10 ? 1 : n == 11 ? 3 : 0; };
    in.pml_judge_z = judge(num_pml[0]);
    in.pml_judge_y = judge(num_pml[1]);
    in.pml_judge_x = judge(num_pml[2]);
    in.pore.q = r.d(); in.pore.porosity = r.d(); in.pore.resistivity = r.d(); r.skip();
    set_zk(in.pore, in.Aav, in.gamma, in.P0);
    const double rho = in.gamma * in.P0 / 340.29 / 340.29;
    in.Z_inf = rho * 340.29 * in.pore.q / in.pore.porosity;
    in.tau = in.gamma * rho * in.pore.q * in.pore.q / in.pore.resistivity / in.pore.porosity;
    for (double& v : in.source) v = r.d();
    for (double& v : in.receiver) v = r.d();
    r.skip();
    in.dt = r.d(); r.skip();
    in.dx = r.d(); in.dy = r.d(); in.dz = r.d(); r.skip();
    r.i(); r.i(); r.i(); r.skip();  // MPI process grid: one device-resident domain here
    r.skip(); r.skip();
    in.restart = r.i(); in.restart_out = r.i(); in.restart_infile = r.word();
    r.skip(); r.skip();
    in.curve_judge = r.i();
    for (double& v : in.curve) v = r.d();
    in.curve_points = r.i(); r.skip();
    for (ZKParams* z : {&in.hill, &in.canopy, &in.trunk}) {
        z->q = r.d(); z->porosity = r.d(); z->resistivity = r.d(); r.skip();
        set_zk(*z, in.Aav, in.gamma, in.P0);
    }
    for (double& v : in.hill_box) v = r.d();
    r.skip();
    r.skip(); r.skip();
    in.has_pore = (in.south == BT_POROUS);
    if (in.has_pore) { in.pdx = r.d(); in.pdy = r.d(); in.pdz = r.d(); r.skip(); }
    if (r.fail) return "malformed " + dir + "/input.txt";
    std::string e = read_axes(dir, "coordi_air", in.air);
    if (!e.empty()) return e;
    if (in.has_pore) {
        e = read_axes(dir, "coordi_pore", in.pore_axes);
        if (!e.empty()) return e;
    }
    // terrain-following grid: no counterpart in the reference (its cross
    // metrics are fixed at zero, calculation_2D.cpp:102-104)
    std::string tt;
    if (slurp(dir + "/terrain.dat", tt)) {
        Reader t{tt};
        const int n = t.i();
        if (t.fail || n != in.air.JMAX) return "terrain.dat must start with the Y node count of coordi_air2.dat";
        in.terrain.resize(static_cast<size_t>(n));
        for (double& v : in.terrain) v = t.d();
        if (t.fail) return "malformed " + dir + "/terrain.dat";
    }
    if (in.velocity_method == 7 && slurp(dir + "/logwind.dat", tt)) {
        Reader t{tt};
        in.wind_kappa = t.d();
        in.wind_z0 = t.d();
        if (t.fail || !(in.wind_kappa > 0.0) || !(in.wind_z0 > 0.0)) return "logwind.dat must hold kappa > 0 and z0 > 0";
    }
    if (slurp(dir + "/advection.dat", tt)) {
        Reader t{tt};
        const std::string w = t.word();
        if (w == "upwind") in.upwind_advection = true;
        else if (w != "reference") return "advection.dat must hold 'upwind' or 'reference'";
    }
    if (slurp(dir + "/tdbc_ground.dat", tt)) {
        Reader t{tt};
        in.g_zinf = t.d();
        in.g_tau = t.d();
        bool bad = false;
        for (double& v : in.g_a) { v = t.d(); bad = bad || !(v >= 0.0); }
        for (double& v : in.g_r) { v = t.d(); bad = bad || !(v >= 0.0); }
        if (t.fail || bad || !(in.g_zinf > 0.0) || !(in.g_tau > 0.0))
            return "tdbc_ground.dat must hold Zinf > 0, tau > 0, six a >= 0 and six r >= 0";
        in.ground_tdbc = true;
    }
    return "";
}

}  // namespace fdtd
