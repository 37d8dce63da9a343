// extern "C" boundary of the B200 FDTD path (declarations: include/fdtd_b200.h).
// Maps C++ exceptions to status codes and keeps a per-thread error message.
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include "../../include/fdtd_b200.h"
#include "../../include/fdtd_surrogate.h"
#include "fdtd_solver.hpp"
#include "mlp.hpp"

struct fdtd_solver {
    fdtd::Solver* s;
};

struct fdtd_ensemble {
    fdtd::Ensemble* e;
};

struct fdtd_net {
    fdtd::mlp::Net* n;
};

namespace {
thread_local std::string g_last_error;

template <typename F>
int guard(F&& f) {
    try {
        f();
        return FDTD_OK;
    } catch (const fdtd::SolverError& e) {
        g_last_error = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return FDTD_ERR_CUDA;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return FDTD_ERR_ARG;
    }
}

int bad(const char* msg) {
    g_last_error = msg;
    return FDTD_ERR_ARG;
}
}  // namespace

namespace fdtd {
// lets entry points outside this file report through fdtd_last_error()
void set_last_error(const char* msg) { g_last_error = msg; }
}  // namespace fdtd

extern "C" {

const char* fdtd_last_error(void) { return g_last_error.c_str(); }

int fdtd_create(const char* case_dir, int precision, int device, fdtd_solver** out) {
    if (!case_dir || !out) return bad("null argument");
    *out = nullptr;
    return guard([&] {
        fdtd::Solver* s = new fdtd::Solver(case_dir, precision, device);
        *out = new fdtd_solver{s};
    });
}

int fdtd_destroy(fdtd_solver* h) {
    if (!h) return FDTD_OK;
    int rc = guard([&] { delete h->s; });
    delete h;
    return rc;
}

int fdtd_dims(const fdtd_solver* h, int* dims) {
    if (!h || !dims) return bad("null argument");
    return guard([&] {
        const auto d = h->s->dims();
        for (int q = 0; q < FDTD_NDIMS; ++q) dims[q] = d[q];
    });
}

int fdtd_set_receivers(fdtd_solver* h, int n, const double* xyz, int* idx_out) {
    if (!h || (n > 0 && !xyz) || n < 0) return bad("bad receiver arguments");
    return guard([&] {
        std::vector<double> v(xyz, xyz + 3 * n);
        const std::vector<int> idx = h->s->set_receivers(v);
        if (idx_out) std::memcpy(idx_out, idx.data(), sizeof(int) * idx.size());
    });
}

int fdtd_reset(fdtd_solver* h, int horizon) {
    if (!h) return bad("null handle");
    return guard([&] { h->s->reset(horizon); });
}

int fdtd_run(fdtd_solver* h, int nsteps, double* rec_out) {
    if (!h || nsteps < 0) return bad("bad run arguments");
    return guard([&] { h->s->run(nsteps, rec_out); });
}

int fdtd_advance(fdtd_solver* h, int nsteps, double* rec_out) {
    if (!h || nsteps < 0) return bad("bad advance arguments");
    int taken = 0;
    int rc = guard([&] { taken = h->s->advance(nsteps, rec_out); });
    if (rc == FDTD_OK && taken < nsteps) {
        g_last_error = "time loop reached its horizon";
        return FDTD_ERR_STATE;
    }
    return rc;
}

int fdtd_step_pressure(fdtd_solver* h) {
    if (!h) return bad("null handle");
    return guard([&] { h->s->step_pressure(); });
}

int fdtd_step_velocity(fdtd_solver* h) {
    if (!h) return bad("null handle");
    return guard([&] { h->s->step_velocity(); });
}

int fdtd_get_field(fdtd_solver* h, int medium, int comp, double* out) {
    if (!h || !out) return bad("null argument");
    return guard([&] { h->s->get_field(medium, comp, out); });
}

int fdtd_set_field(fdtd_solver* h, int medium, int comp, const double* in) {
    if (!h || !in) return bad("null argument");
    return guard([&] { h->s->set_field(medium, comp, in); });
}

int fdtd_get_psi(fdtd_solver* h, double* out) {
    if (!h || !out) return bad("null argument");
    return guard([&] { h->s->get_psi(out); });
}

int fdtd_get_ground_psi(fdtd_solver* h, double* out) {
    if (!h || !out) return bad("null argument");
    return guard([&] { h->s->get_ground_psi(out); });
}

int fdtd_get_slab(fdtd_solver* h, int s, int comp, double* out, int* dims) {
    if (!h || !dims) return bad("null argument");
    int present = 0;
    int rc = guard([&] { present = h->s->get_slab(s, comp, out, dims); });
    return rc == FDTD_OK ? present : rc;
}

size_t fdtd_state_elems(const fdtd_solver* h) { return h ? h->s->state_elems() : 0; }

int fdtd_copy_state(fdtd_solver* h, int dir, void* host) {
    if (!h || !host || (dir != 0 && dir != 1)) return bad("bad copy_state arguments");
    return guard([&] { h->s->copy_state(dir, host); });
}

int fdtd_set_tiling(fdtd_solver* h, int rows_per_block, int planes_per_block, int threads_per_block, int vector_width,
                    int ring_stages) {
    if (!h) return bad("null handle");
    return guard([&] { h->s->set_tiling(rows_per_block, planes_per_block, threads_per_block, vector_width, ring_stages); });
}

int fdtd_set_tile_shape(fdtd_solver* h, int kind, int rows, int vectors, int planes, int ring_stages) {
    if (!h) return bad("null handle");
    return guard([&] { h->s->set_tile_shape(kind, rows, vectors, planes, ring_stages); });
}

int fdtd_get_tile_shape(const fdtd_solver* h, int* out) {
    if (!h || !out) return bad("null argument");
    return guard([&] {
        const auto t = h->s->tile_shape();
        for (int q = 0; q < 19; ++q) out[q] = t[q];
    });
}

int fdtd_set_block_trace(fdtd_solver* h, int on) {
    if (!h) return bad("null handle");
    return guard([&] { h->s->set_block_trace(on != 0); });
}

int fdtd_get_block_trace(fdtd_solver* h, unsigned long long* out) {
    if (!h || !out) return bad("null argument");
    return guard([&] { h->s->get_block_trace(out); });
}

int fdtd_autotune(fdtd_solver* h, int nsteps, int* best) {
    if (!h || !best || nsteps <= 0) return bad("bad autotune arguments");
    return guard([&] {
        const auto b = h->s->autotune(nsteps);
        for (int q = 0; q < 5; ++q) best[q] = b[q];
    });
}

long long fdtd_launch_count(const fdtd_solver* h) { return h ? h->s->launch_count() : 0; }

int fdtd_last_device_ms(const fdtd_solver* h, double* ms) {
    if (!h || !ms) return bad("null argument");
    *ms = h->s->last_device_ms();
    return FDTD_OK;
}

}  // extern "C"

int fdtd_fft(int device, const double* traces, int nrec, int nt, int fft_m, double* re, double* im) {
    if (!traces || !re || !im) return bad("null argument");
    return guard([&] { fdtd::fft_forward(device, traces, nrec, nt, fft_m, re, im); });
}

int fdtd_spectrum(int device, const double* traces, int nrec, int nt, int fft_m, long long k0, long long nk,
                  double* mag) {
    if (!traces || !mag) return bad("null argument");
    return guard([&] { fdtd::spectrum_bins(device, traces, nrec, nt, fft_m, static_cast<long>(k0), static_cast<long>(nk), mag); });
}

int fdtd_band_levels(int device, const double* traces, int nrec, int nt, int fft_m, double dt, int nband,
                     const double* fc, double* levels_db) {
    if (!traces || !fc || !levels_db) return bad("null argument");
    return guard([&] { fdtd::band_levels(device, traces, nrec, nt, fft_m, dt, nband, fc, levels_db); });
}

int fdtd_save_restart(fdtd_solver* h, const char* path) {
    if (!h || !path) return bad("null argument");
    return guard([&] { h->s->save_restart(path); });
}

int fdtd_load_restart(fdtd_solver* h, const char* path, int reference_semantics) {
    if (!h || !path) return bad("null argument");
    return guard([&] { h->s->load_restart(path, reference_semantics != 0); });
}

int fdtd_write_contour(fdtd_solver* h, const char* path, int format) {
    if (!h || !path) return bad("null argument");
    return guard([&] { h->s->write_contour(path, format); });
}

int fdtd_get_receivers(fdtd_solver* h, int first_step, int nsteps, double* out) {
    if (!h || (!out && nsteps > 0)) return bad("null argument");
    return guard([&] { h->s->get_receivers(first_step, nsteps, out); });
}

int fdtd_set_wait_limit(fdtd_solver* h, long long polls) {
    if (!h) return bad("null argument");
    return guard([&] { h->s->set_wait_limit(polls); });
}

int fdtd_ensemble_create(fdtd_solver* const* members, int n, fdtd_ensemble** out) {
    if (!members || !out || n < 1) return bad("bad ensemble arguments");
    *out = nullptr;
    return guard([&] {
        std::vector<fdtd::Solver*> m;
        for (int i = 0; i < n; ++i) {
            if (!members[i]) throw fdtd::SolverError{FDTD_ERR_ARG, "null ensemble member"};
            m.push_back(members[i]->s);
        }
        fdtd::Ensemble* e = new fdtd::Ensemble(m);
        *out = new fdtd_ensemble{e};
    });
}

int fdtd_ensemble_destroy(fdtd_ensemble* e) {
    if (!e) return FDTD_OK;
    const int rc = guard([&] { delete e->e; });
    delete e;
    return rc;
}

int fdtd_ensemble_advance(fdtd_ensemble* e, int nsteps, int* taken) {
    if (!e || nsteps < 0) return bad("bad ensemble advance arguments");
    return guard([&] {
        const int n = e->e->advance(nsteps);
        if (taken) *taken = n;
    });
}

int fdtd_ensemble_autotune(fdtd_ensemble* e, int nsteps, int* best) {
    if (!e || !best || nsteps <= 0) return bad("bad autotune arguments");
    return guard([&] {
        const auto b = e->e->autotune(nsteps);
        best[0] = b[0];
        best[1] = b[1];
    });
}

int fdtd_ensemble_info(const fdtd_ensemble* e, long long* info) {
    if (!e || !info) return bad("null argument");
    return guard([&] {
        const auto s = e->e->shape();
        info[0] = e->e->launch_count();
        info[1] = s[0];
        info[2] = s[1];
    });
}

int fdtd_ensemble_set_mode(fdtd_ensemble* e, int mode) {
    if (!e) return bad("null argument");
    return guard([&] { e->e->set_mode(mode); });
}

int fdtd_ensemble_last_device_ms(const fdtd_ensemble* e, double* ms) {
    if (!e || !ms) return bad("null argument");
    *ms = e->e->last_device_ms();
    return FDTD_OK;
}

// ------------------------------------------------------------- surrogate
extern "C" {

int fdtd_tc_gemm(int device, int epilogue, int M, int N, int K, const void* A, const void* B, const float* bias,
                 const void* mask, void* out, void* outT, void* stream) {
    return guard([&] { fdtd::mlp::gemm(device, epilogue, M, N, K, A, B, bias, mask, out, outT, stream); });
}

int fdtd_net_create(int device, int n_in, int width, int hidden, int n_out, int batch, unsigned long long seed,
                    fdtd_net** out) {
    if (!out) return bad("null argument");
    *out = nullptr;
    return guard([&] {
        auto* n = new fdtd::mlp::Net(device, n_in, width, hidden, n_out, batch, seed);
        *out = new fdtd_net{n};
    });
}

int fdtd_net_destroy(fdtd_net* h) {
    if (!h) return FDTD_OK;
    const int rc = guard([&] { delete h->n; });
    delete h;
    return rc;
}

int fdtd_net_n_params(const fdtd_net* h, int* n) {
    if (!h || !n) return bad("null argument");
    *n = h->n->n_params();
    return FDTD_OK;
}

int fdtd_net_get_params(const fdtd_net* h, float* out) {
    if (!h || !out) return bad("null argument");
    return guard([&] { h->n->get_params(out); });
}

int fdtd_net_set_params(fdtd_net* h, const float* in) {
    if (!h || !in) return bad("null argument");
    return guard([&] { h->n->set_params(in); });
}

int fdtd_net_set_data(fdtd_net* h, const float* X, const float* T, int n) {
    if (!h || !X || !T) return bad("null argument");
    return guard([&] { h->n->set_data(X, T, n); });
}

int fdtd_net_get_normalization(const fdtd_net* h, float* im, float* is, float* om, float* os) {
    if (!h || !im || !is || !om || !os) return bad("null argument");
    return guard([&] { h->n->get_normalization(im, is, om, os); });
}

int fdtd_net_set_normalization(fdtd_net* h, const float* im, const float* is, const float* om, const float* os) {
    if (!h || !im || !is || !om || !os) return bad("null argument");
    return guard([&] { h->n->set_normalization(im, is, om, os); });
}

int fdtd_net_train(fdtd_net* h, int steps, float lr, float lr_final, float weight_decay, unsigned long long seed,
                   int report, double* loss) {
    if (!h) return bad("null argument");
    return guard([&] {
        const double l = h->n->train(steps, lr, lr_final, seed, report, weight_decay);
        if (loss) *loss = l;
    });
}

int fdtd_net_gradients(fdtd_net* h, float* grad, double* loss) {
    if (!h || !grad) return bad("null argument");
    return guard([&] {
        const double l = h->n->gradients(grad);
        if (loss) *loss = l;
    });
}

int fdtd_net_predict(fdtd_net* h, const float* X, int n, float* Y) {
    if (!h || (n > 0 && (!X || !Y))) return bad("null argument");
    return guard([&] { h->n->predict(X, n, Y); });
}

int fdtd_net_predict_device(fdtd_net* h, const float* X, int n, float* Y, void* stream) {
    if (!h || (n > 0 && (!X || !Y))) return bad("null argument");
    return guard([&] { h->n->predict_device(X, n, Y, stream); });
}

int fdtd_net_ensemble_predict(fdtd_net* const* nets, int members, const float* X, int n, float* mean, float* spread) {
    if (!nets || members < 1 || (n > 0 && (!X || !mean || !spread))) return bad("bad ensemble arguments");
    return guard([&] {
        std::vector<fdtd::mlp::Net*> v;
        for (int m = 0; m < members; ++m) {
            if (!nets[m]) throw fdtd::SolverError{FDTD_ERR_ARG, "null ensemble member"};
            v.push_back(nets[m]->n);
        }
        fdtd::mlp::ensemble_predict(v.data(), members, X, n, mean, spread);
    });
}

int fdtd_ray_features(const float* P, int n, int n_par, int col_hs, int col_hr, int col_range, int n_rec, float* F,
                      void* stream) {
    if (n < 0 || (n > 0 && (!P || !F))) return bad("bad ray-feature arguments");
    return guard([&] {
        fdtd::mlp::ray_features(fdtd::mlp::RayFeatures{n_par, col_hs, col_hr, col_range, n_rec}, P, n, F, stream);
    });
}

int fdtd_net_ensemble_predict_rays(fdtd_net* const* nets, int members, const float* P, int n, int n_par, int col_hs,
                                   int col_hr, int col_range, int n_rec, float* mean, float* spread) {
    if (!nets || members < 1 || (n > 0 && (!P || !mean || !spread))) return bad("bad ensemble arguments");
    return guard([&] {
        std::vector<fdtd::mlp::Net*> v;
        for (int m = 0; m < members; ++m) {
            if (!nets[m]) throw fdtd::SolverError{FDTD_ERR_ARG, "null ensemble member"};
            v.push_back(nets[m]->n);
        }
        fdtd::mlp::ensemble_predict_rays(v.data(), members,
                                         fdtd::mlp::RayFeatures{n_par, col_hs, col_hr, col_range, n_rec}, P, n, mean,
                                         spread);
    });
}

int fdtd_net_set_fused(fdtd_net* h, int on, int* served) {
    if (!h) return bad("null argument");
    return guard([&] {
        const bool ok = h->n->set_fused(on != 0);
        if (served) *served = ok ? 1 : 0;
    });
}

int fdtd_net_info(const fdtd_net* h, long long* launches, double* last_ms) {
    if (!h) return bad("null argument");
    if (launches) *launches = h->n->launches();
    if (last_ms) *last_ms = h->n->last_device_ms();
    return FDTD_OK;
}

}  // extern "C"
