/*
 * Full-precision driver for the UNMODIFIED reference solver (test
 * infrastructure: builds only into oracle/_ref/, never shipped).
 *
 * The reference's own main() (main.cpp:8-26) runs airpore::get_output,
 * which writes receiver p(t) with 6 significant digits
 * (airpore.cpp:522-524) at hard-coded positions (airpore.cpp:431-453).
 * This driver calls the same public/protected members in the same order
 * as the get_output loop (airpore.cpp:539-624):
 *   SetMovingFrame(MF_count); per step: get_pressure() per receiver,
 *   Cal_pressure(); Cal_velocity(); UpdateInitialCond(MF_count)
 * and dumps receivers, final fields, TDBC state and PML integrals as FP64.
 * Contour output, restart files and FFT post-processing are skipped; they
 * do not feed back into the state.
 *
 * Usage: ref_harness <case_dir> [--steps N] [--receivers FILE] [--out FILE]
 *                    [--time WARMUP TIMED]
 *   case_dir holds input.txt and coordi_air{1,2,3}.dat (+ coordi_pore*).
 *   --steps overrides input.txt's time_domain (airpore.cpp:171).
 *   --receivers: text file, one "X Y Z" per line (reference axes).
 *   --time: no dump; prints one JSON line with ms per step.
 *   --restart-out FILE: after the run, write the reference's restart file
 *     (the header line of airpore::Save_restart, airpore.cpp:686-689, then
 *     airpore::save_restartfile, airpore.cpp:782-796) for the step reached.
 *   --contour-out FILE: after the run, the pressure contour of the last step
 *     as airpore::get_data_contour writes it (airpore.cpp:1014-1056, with the
 *     reference's own operator<<, calculation_2D.cpp:1171-1190), to FILE
 *     instead of its hard-coded cluster path.
 *   --restart-in FILE: before the run, load a restart file with the
 *     reference's airpore::input_restartfile (airpore.cpp:798-863, the
 *     timer as in get_output, airpore.cpp:499-504); the run then takes
 *     --steps further steps. Only without a moving frame (the reference does
 *     not store the frame count). The reference passes its short restart
 *     name to the porous reader (airpore.cpp:869) and keeps names in
 *     char[20]; here both readers get a copy named rs_in.dat in the case
 *     directory.
 */
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>
#include <unistd.h>

#define private public
#define protected public
#include "airpore.h"
#include "calculation_2D.h"
#include "air.h"
#include "porous.h"
#undef private
#undef protected

namespace {

struct Rec { double x, y, z; int i, j, k; };

void put_i32(FILE *f, int32_t v) { fwrite(&v, 4, 1, f); }

void put_field(FILE *f, double ***a, int I, int J, int K)
{
    std::vector<double> row((size_t)K);
    for (int i = 0; i < I; ++i)
        for (int j = 0; j < J; ++j) {
            for (int k = 0; k < K; ++k) row[k] = a[i][j][k];
            fwrite(row.data(), 8, (size_t)K, f);
        }
}

void put_slab(FILE *f, int id, double ***qu, double ***qv, double ***qw, double ***qp,
              int d0, int d1, int d2)
{
    put_i32(f, id); put_i32(f, d0); put_i32(f, d1); put_i32(f, d2);
    put_field(f, qu, d0, d1, d2);
    put_field(f, qv, d0, d1, d2);
    put_field(f, qw, d0, d1, d2);
    put_field(f, qp, d0, d1, d2);
}

/* One FB step exactly as dispatched at airpore.cpp:589-614. */
void one_step(airpore *ap, int MF_count)
{
    scheme_list s = ap->scheme;
    if (s == FB_p_v || s == LeapTrap) {
        ap->Cal_pressure();
        ap->Cal_velocity();
    } else if (s == FB_v_p) {
        ap->Cal_velocity();
        ap->Cal_pressure();
    } else {
        ap->Cal_pressure();
        ap->Cal_velocity();
        ap->UpdateInitialCond(MF_count);
        ap->Cal_pressure();
        ap->Cal_velocity();
    }
    ap->UpdateInitialCond(MF_count);
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s case_dir [--steps N] [--receivers F] [--out F] [--time W K]\n", argv[0]);
        return 2;
    }
    std::string case_dir = argv[1], rec_file, out_file = "ref_out.bin", restart_out, restart_in, contour_out;
    long steps_override = -1;
    int time_w = -1, time_k = -1;
    for (int a = 2; a < argc; ++a) {
        std::string s = argv[a];
        if (s == "--steps" && a + 1 < argc) steps_override = std::atol(argv[++a]);
        else if (s == "--receivers" && a + 1 < argc) rec_file = argv[++a];
        else if (s == "--out" && a + 1 < argc) out_file = argv[++a];
        else if (s == "--time" && a + 2 < argc) { time_w = std::atoi(argv[++a]); time_k = std::atoi(argv[++a]); }
        else if (s == "--restart-out" && a + 1 < argc) restart_out = argv[++a];
        else if (s == "--restart-in" && a + 1 < argc) restart_in = argv[++a];
        else if (s == "--contour-out" && a + 1 < argc) contour_out = argv[++a];
        else { std::fprintf(stderr, "bad argument %s\n", s.c_str()); return 2; }
    }
    /* Resolve output/receiver paths before changing directory. */
    auto absolutize = [](const std::string &p) {
        if (p.empty() || p[0] == '/') return p;
        char buf[4096];
        if (!getcwd(buf, sizeof buf)) return p;
        return std::string(buf) + "/" + p;
    };
    rec_file = absolutize(rec_file);
    out_file = absolutize(out_file);
    restart_out = absolutize(restart_out);
    restart_in = absolutize(restart_in);
    contour_out = absolutize(contour_out);

    std::vector<Rec> recs;
    if (!rec_file.empty()) {
        std::ifstream rf(rec_file);
        Rec r{};
        while (rf >> r.x >> r.y >> r.z) recs.push_back(r);
    }
    if (chdir(case_dir.c_str()) != 0) { std::perror("chdir"); return 2; }

    /* Silence the reference's progress prints (cout) to keep the driver fast. */
    std::ofstream devnull("/dev/null");
    std::streambuf *old_cout = std::cout.rdbuf(devnull.rdbuf());

    char input_name[] = "input.txt";
    airpore *ap = new airpore(input_name);
    ap->mpi_rank = 0;
    ap->mpi_size = 1;
    if (steps_override >= 0) ap->time_domain = (int)steps_override;
    if (time_w >= 0) ap->time_domain = time_w + time_k;
    ap->MPI_Initialize();
    ap->SetInitialCond();

    calculation_2D *A = ap->AirMedia;
    int IMAXw = A->get_whole_IMAX(), JMAXw = A->get_whole_JMAX(), KMAXw = A->get_whole_KMAX();
    /* Receiver index search and out-of-domain rule: airpore.cpp:431-457. */
    for (auto &r : recs) {
        int ii = 0, jj = 0, kk = 0;
        Position pos; pos.x = r.x; pos.y = r.y; pos.z = r.z;
        A->get_position(ii, jj, kk, pos);
        if (ii == 0 && jj == 0 && kk == 0) { ii = 1; jj = 1; kk = 1; }
        if (ii > IMAXw || jj > JMAXw || kk > KMAXw) { ii = 1; jj = 1; kk = 1; }
        r.i = ii; r.j = jj; r.k = kk;
    }

    int restart_index = 0;
    if (!restart_in.empty()) {
        if (ap->move_frame.Judge == 1) { std::fprintf(stderr, "--restart-in needs a case without moving frame\n"); return 2; }
        std::ifstream hin(restart_in, std::ios::in | std::ios::binary);
        int re_size = 0, re_rank = 0;
        hin >> re_size >> re_rank >> restart_index;
        hin.ignore(100, '\n');
        int pos = (int)hin.tellg();
        hin.close();
        // the reference keeps the name in char[20] (airpore.h:30): read a copy
        // under a short name in the case directory (the working directory)
        {
            std::ifstream src(restart_in, std::ios::binary);
            std::ofstream dst("rs_in.dat", std::ios::binary | std::ios::trunc);
            dst << src.rdbuf();
        }
        std::snprintf(ap->restart_infile1, sizeof ap->restart_infile1, "%s", "rs_in.dat");
        std::snprintf(ap->restart_infile, sizeof ap->restart_infile, "%s", "rs_in.dat");
        ap->input_restartfile(&pos);
        A->Set_Timer(restart_index);
    }

    const int time_domain = ap->time_domain;
    std::vector<double> rec_out((size_t)time_domain * (recs.empty() ? 1 : recs.size()), 0.0);
    MovingFrame &mf = ap->move_frame;
    const int JMAX = JMAXw;
    const double dy = ap->AirStep.diff_y, dt = ap->AirStep.diff_t, c0 = ap->AirPara.sound_speed;
    int MF_count = 0, temp_time = 0, index_pressure = 0, MF_limit = 0;
    auto t_start = std::chrono::steady_clock::now();
    auto t_end = t_start;

    /* Frame loop: airpore.cpp:539-624. */
    do {
        if (MF_count == (int)((JMAX - mf.JMAX) / (mf.lead_DJ - 1) + 1.e-6) || (JMAX == mf.JMAX)) {
            MF_limit = time_domain - temp_time;
        } else if (MF_count == 0) {
            MF_limit = (int)((mf.JMAX - 1) * dy / c0 / dt * mf.ratio);
        } else {
            MF_limit = (int)((mf.trail_DJ - 1) * dy / c0 / dt);
            double MF_lefttime1 = 0.0, MF_lefttime2 = 0.0;
            if (MF_count % 10 == 0) {
                MF_lefttime1 = (mf.trail_DJ - 1) * dy / c0 / dt - MF_limit;
                MF_lefttime1 = MF_lefttime1 * 10.0;
            }
            if (MF_count % 100 == 0) {
                MF_lefttime2 = (mf.trail_DJ - 1) * dy / c0 / dt - MF_limit;
                MF_lefttime2 = MF_lefttime2 * 100 - int(MF_lefttime2 * 10) * 10;
            }
            MF_limit = MF_limit + int(MF_lefttime1) + int(MF_lefttime2);
            if ((temp_time + MF_limit) > time_domain) MF_limit = time_domain - temp_time;
        }
        ap->SetMovingFrame(MF_count);
        for (int n = 0; n < MF_limit; n++) {
            if (time_w >= 0 && index_pressure == time_w) t_start = std::chrono::steady_clock::now();
            index_pressure = index_pressure + 1;
            for (size_t r = 0; r < recs.size(); ++r) {
                double temp = A->get_pressure(recs[r].i, recs[r].j, recs[r].k, MF_count);
                if (std::fabs(temp) < 1.0e-100) temp = 0.0;
                /* frame 0 may run past time_domain (airpore.cpp:545); keep the buffer in bounds */
                if (index_pressure <= time_domain) rec_out[(size_t)(index_pressure - 1) * recs.size() + r] = temp;
            }
            one_step(ap, MF_count);
        }
        MF_count = MF_count + 1;
        temp_time = MF_limit + temp_time;
    } while ((MF_count <= (int)((JMAX - mf.JMAX) / (mf.lead_DJ - 1) + 1.e-6)) && (temp_time < time_domain) &&
             mf.Judge == 1);
    t_end = std::chrono::steady_clock::now();
    if (!contour_out.empty()) {
        ap->mpisend_data_contour(MF_count > 0 ? MF_count - 1 : 0);
        std::ofstream fp_p_t(contour_out, std::ios::out | std::ios::trunc | std::ios::binary);
        fp_p_t.setf(std::ios::scientific, std::ios::floatfield);
        fp_p_t.precision(6);
        if (ap->air_boundary.air_south == rigid || ap->air_boundary.air_south == absorbing) {
            fp_p_t << "VARIABLES = \"X\", \"Y\", \"Z\", \"P\"" << std::endl;
            fp_p_t << "ZONE T = \"Air Zone\",";
            fp_p_t << *ap->AirMedia;
        } else {
            fp_p_t << "ZONE T = \"Air Zone\",";
            fp_p_t << *ap->AirMedia;
            fp_p_t << "ZONE T = \"south pore Zone\",";
            fp_p_t << *ap->south_pore;
        }
    }
    if (!restart_out.empty()) {
        std::ofstream hout(restart_out, std::ios::out | std::ios::trunc | std::ios::binary);
        hout << ap->mpi_size << " " << ap->mpi_rank << " " << restart_index + index_pressure << std::endl;
        hout.close();
        std::vector<char> name(restart_out.begin(), restart_out.end());
        name.push_back('\0');
        ap->save_restartfile(name.data());
    }
    std::cout.rdbuf(old_cout);

    if (time_w >= 0) {
        double ms = std::chrono::duration<double, std::milli>(t_end - t_start).count();
        long nodes = (long)A->mpi_IMAX * A->mpi_JMAX * A->mpi_KMAX;
        long pore_nodes = 0;
        if (ap->air_boundary.air_south == porous_media && ap->south_pore)
            pore_nodes = (long)ap->south_pore->mpi_IMAX * ap->south_pore->mpi_JMAX * ap->south_pore->mpi_KMAX;
        std::printf("{\"ms_per_step\": %.6f, \"steps\": %d, \"warmup\": %d, \"air_nodes\": %ld, \"pore_nodes\": %ld}\n",
                    time_k > 0 ? ms / time_k : 0.0, time_k, time_w, nodes, pore_nodes);
        return 0;
    }

    FILE *f = std::fopen(out_file.c_str(), "wb");
    if (!f) { std::perror("fopen"); return 3; }
    air *AA = static_cast<air *>(A);
    int has_pore = (ap->air_boundary.air_south == porous_media) ? 1 : 0;
    calculation_2D *P = has_pore ? ap->south_pore : nullptr;
    struct SlabDesc { int id; double ***u, ***v, ***w, ***p; int d0, d1, d2; };
    std::vector<SlabDesc> slabs;
    if (AA->mpi_IMAX1) slabs.push_back({0, AA->Qux1, AA->Qvx1, AA->Qwx1, AA->Qpx1, AA->mpi_IMAX1, A->mpi_JMAX, A->mpi_KMAX});
    if (AA->mpi_IMAX2) slabs.push_back({1, AA->Qux2, AA->Qvx2, AA->Qwx2, AA->Qpx2, AA->mpi_IMAX2, A->mpi_JMAX, A->mpi_KMAX});
    if (AA->mpi_JMAX1) slabs.push_back({2, AA->Quy1, AA->Qvy1, AA->Qwy1, AA->Qpy1, A->mpi_IMAX, AA->mpi_JMAX1, A->mpi_KMAX});
    if (AA->mpi_JMAX2) slabs.push_back({3, AA->Quy2, AA->Qvy2, AA->Qwy2, AA->Qpy2, A->mpi_IMAX, AA->mpi_JMAX2, A->mpi_KMAX});
    if (AA->mpi_KMAX1) slabs.push_back({4, AA->Quz1, AA->Qvz1, AA->Qwz1, AA->Qpz1, A->mpi_IMAX, A->mpi_JMAX, AA->mpi_KMAX1});
    if (AA->mpi_KMAX2) slabs.push_back({5, AA->Quz2, AA->Qvz2, AA->Qwz2, AA->Qpz2, A->mpi_IMAX, A->mpi_JMAX, AA->mpi_KMAX2});

    std::fwrite("FDTDREF1", 1, 8, f);
    put_i32(f, (int32_t)recs.size());
    put_i32(f, time_domain);
    put_i32(f, A->mpi_IMAX); put_i32(f, A->mpi_JMAX); put_i32(f, A->mpi_KMAX);
    put_i32(f, has_pore);
    put_i32(f, P ? P->mpi_IMAX : 0); put_i32(f, P ? P->mpi_JMAX : 0); put_i32(f, P ? P->mpi_KMAX : 0);
    put_i32(f, (int32_t)slabs.size());
    for (auto &r : recs) { put_i32(f, r.i); put_i32(f, r.j); put_i32(f, r.k); }
    if (!recs.empty()) std::fwrite(rec_out.data(), 8, rec_out.size(), f);
    put_field(f, A->p_n, A->mpi_IMAX, A->mpi_JMAX, A->mpi_KMAX);
    put_field(f, A->u_n, A->mpi_IMAX, A->mpi_JMAX, A->mpi_KMAX);
    put_field(f, A->v_n, A->mpi_IMAX, A->mpi_JMAX, A->mpi_KMAX);
    put_field(f, A->w_n, A->mpi_IMAX, A->mpi_JMAX, A->mpi_KMAX);
    if (P) {
        put_field(f, P->p_n, P->mpi_IMAX, P->mpi_JMAX, P->mpi_KMAX);
        put_field(f, P->u_n, P->mpi_IMAX, P->mpi_JMAX, P->mpi_KMAX);
        put_field(f, P->v_n, P->mpi_IMAX, P->mpi_JMAX, P->mpi_KMAX);
        put_field(f, P->w_n, P->mpi_IMAX, P->mpi_JMAX, P->mpi_KMAX);
    }
    put_field(f, A->Psi, A->mpi_IMAX, A->mpi_KMAX, A->Ns);
    for (auto &s : slabs) put_slab(f, s.id, s.u, s.v, s.w, s.p, s.d0, s.d1, s.d2);
    std::fclose(f);
    return 0;
}
