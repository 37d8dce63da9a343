// Drives a case through the C++ host classes the way the reference's
// main.cpp drives airpore (airpore(input) -> get_output), then through the
// half-step members in the order of airpore.cpp:589-614, and writes what the
// test compares with the oracle:
//   <out>.rec     receivers [step][receiver] (FP64, native byte order)
//   <out>.p       final air pressure [i][j][k]
//   <out>.pore_p  final porous pressure (porous ground only)
//   <out>.half_p  final air pressure after the same steps as half steps
// Usage: mirror_driver <case_dir> <receivers.txt> <nsteps> <out> [f32]
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "airpore_b200.hpp"

static void dump(const std::string& path, const std::vector<double>& v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(double)));
}

int main(int argc, char** argv) {
    if (argc < 5) {
        std::cerr << "usage: mirror_driver <case_dir> <receivers.txt> <nsteps> <out> [f32]\n";
        return 2;
    }
    const std::string dir = argv[1], out = argv[4];
    const int nsteps = std::stoi(argv[3]);
    const b200::Precision prec = (argc > 5 && std::string(argv[5]) == "f32") ? b200::FP32 : b200::FP64;
    std::vector<b200::Position> rec;
    {
        std::ifstream f(argv[2]);
        b200::Position p;
        while (f >> p.x >> p.y >> p.z) rec.push_back(p);
    }
    try {
        b200::airpore a(dir, prec);
        a.MPI_Initialize();
        a.set_receivers(rec);
        a.get_output(nsteps);
        dump(out + ".rec", a.receivers());
        dump(out + ".p", a.AirMedia->field('p'));
        if (a.south_pore) dump(out + ".pore_p", a.south_pore->field('p'));
        // the reference's per-step member calls (airpore.cpp:589-614)
        a.SetInitialCond(nsteps);
        for (int n = 0; n < nsteps; ++n) {
            a.Cal_pressure();
            a.AirMedia->Update_PML_Qp();
            a.Cal_velocity();
            a.AirMedia->Update_PML_Qvw();
            a.UpdateInitialCond(0);
        }
        dump(out + ".half_p", a.AirMedia->field('p'));
        std::printf("{\"steps\": %d, \"receivers\": %d, \"I\": %d, \"J\": %d, \"K\": %d, \"porous\": %d}\n", nsteps,
                    a.n_receivers(), a.AirMedia->get_whole_IMAX(), a.AirMedia->get_whole_JMAX(),
                    a.AirMedia->get_whole_KMAX(), a.south_pore ? 1 : 0);
    } catch (const b200::Error& e) {
        std::fprintf(stderr, "fdtd error %d: %s\n", e.code, e.what());
        return 3;
    }
    return 0;
}
