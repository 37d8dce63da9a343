// C++ host classes over the C ABI: see airpore_b200.hpp.
#include "airpore_b200.hpp"

namespace b200 {
namespace {

void check(int rc) {
    if (rc != FDTD_OK) throw Error(rc, fdtd_last_error());
}

int comp_index(char c) {
    switch (c) {
        case 'p': return 0;
        case 'u': return 1;
        case 'v': return 2;
        case 'w': return 3;
        default: throw Error(FDTD_ERR_ARG, std::string("field component must be p, u, v or w, not ") + c);
    }
}

}  // namespace

// ------------------------------------------------------------ calculation_2D
calculation_2D::calculation_2D(fdtd_solver* h, int medium) : h_(h), medium_(medium) {
    int d[FDTD_NDIMS];
    check(fdtd_dims(h, d));
    if (medium == 0) {
        I_ = d[0]; J_ = d[1]; K_ = d[2];
    } else {
        I_ = d[4]; J_ = d[5]; K_ = d[6];
    }
}

std::vector<double> calculation_2D::field(char comp) const {
    std::vector<double> out(static_cast<size_t>(I_) * J_ * K_);
    check(fdtd_get_field(h_, medium_, comp_index(comp), out.data()));
    return out;
}

void calculation_2D::set_field(char comp, const std::vector<double>& v) {
    if (v.size() != static_cast<size_t>(I_) * J_ * K_) throw Error(FDTD_ERR_ARG, "field size differs from the grid");
    check(fdtd_set_field(h_, medium_, comp_index(comp), v.data()));
}

double calculation_2D::get_pressure(int ii, int jj, int kk) const {
    if (ii <= 0 || ii >= I_ - 1 || jj <= 0 || jj >= J_ - 1 || kk <= 0 || kk >= K_ - 1) return 0.0;
    const std::vector<double> p = field('p');
    return p[(static_cast<size_t>(ii) * J_ + jj) * K_ + kk];
}

// ----------------------------------------------------------------------- air
std::vector<double> air::pml_slab(int s, char comp, std::array<int, 3>* dims) const {
    int d[3] = {0, 0, 0};
    const int rc = fdtd_get_slab(h_, s, comp_index(comp), nullptr, d);
    if (rc < 0) check(rc);
    if (dims) *dims = {d[0], d[1], d[2]};
    if (rc == 0) return {};
    std::vector<double> out(static_cast<size_t>(d[0]) * d[1] * d[2]);
    const int rc2 = fdtd_get_slab(h_, s, comp_index(comp), out.data(), d);
    if (rc2 < 0) check(rc2);
    return out;
}

std::vector<double> air::psi() const {
    std::vector<double> out(static_cast<size_t>(I_) * K_ * 6);
    check(fdtd_get_psi(h_, out.data()));
    return out;
}

std::vector<double> air::ground_psi() const {
    std::vector<double> out(static_cast<size_t>(I_) * J_ * 6);
    check(fdtd_get_ground_psi(h_, out.data()));
    return out;
}

// ------------------------------------------------------------------- airpore
airpore::airpore(const std::string& case_dir, Precision precision, int device) : device_(device) {
    check(fdtd_create(case_dir.c_str(), precision, device, &h_));
    try {
        check(fdtd_dims(h_, dims_.data()));
        air_ = std::make_unique<air>(h_);
        AirMedia = air_.get();
        if (dims_[3]) {
            pore_ = std::make_unique<porous>(h_);
            south_pore = pore_.get();
        }
    } catch (...) {
        fdtd_destroy(h_);
        throw;
    }
}

airpore::~airpore() {
    if (h_) fdtd_destroy(h_);
}

void airpore::SetInitialCond(int horizon) {
    check(fdtd_reset(h_, horizon));
    rec_.clear();
}

void airpore::Cal_pressure() { check(fdtd_step_pressure(h_)); }

void airpore::Cal_velocity() { check(fdtd_step_velocity(h_)); }

std::vector<std::array<int, 3>> airpore::set_receivers(const std::vector<Position>& r) {
    std::vector<double> xyz;
    for (const Position& q : r) {
        xyz.push_back(q.x);
        xyz.push_back(q.y);
        xyz.push_back(q.z);
    }
    std::vector<int> idx(3 * r.size());
    check(fdtd_set_receivers(h_, static_cast<int>(r.size()), xyz.data(), idx.data()));
    nrec_ = static_cast<int>(r.size());
    std::vector<std::array<int, 3>> out(r.size());
    for (size_t q = 0; q < r.size(); ++q) out[q] = {idx[3 * q], idx[3 * q + 1], idx[3 * q + 2]};
    return out;
}

void airpore::get_output(int nsteps) {
    const int n = nsteps > 0 ? nsteps : time_domain();
    rec_.assign(static_cast<size_t>(n) * std::max(nrec_, 1), 0.0);
    check(fdtd_run(h_, n, rec_.data()));
    rec_.resize(static_cast<size_t>(n) * nrec_);
}

void airpore::advance(int nsteps) {
    std::vector<double> r(static_cast<size_t>(nsteps) * std::max(nrec_, 1), 0.0);
    check(fdtd_advance(h_, nsteps, r.data()));
    rec_.insert(rec_.end(), r.begin(), r.begin() + static_cast<size_t>(nsteps) * nrec_);
}

int airpore::steps_taken() const {
    int d[FDTD_NDIMS];
    check(fdtd_dims(h_, d));
    return d[11];
}

std::vector<double> airpore::band_levels(int fft_m, double dt, const std::vector<double>& centres) const {
    if (nrec_ == 0 || rec_.empty()) return {};
    const int nt = static_cast<int>(rec_.size() / nrec_);
    std::vector<double> traces(rec_.size());  // [receiver][step]
    for (int t = 0; t < nt; ++t)
        for (int r = 0; r < nrec_; ++r) traces[static_cast<size_t>(r) * nt + t] = rec_[static_cast<size_t>(t) * nrec_ + r];
    std::vector<double> out(static_cast<size_t>(nrec_) * centres.size());
    check(fdtd_band_levels(device_, traces.data(), nrec_, nt, fft_m, dt, static_cast<int>(centres.size()),
                           centres.data(), out.data()));
    return out;
}

void airpore::Save_restart(const std::string& path) { check(fdtd_save_restart(h_, path.c_str())); }

void airpore::Read_restart(const std::string& path, bool reference_semantics) {
    check(fdtd_load_restart(h_, path.c_str(), reference_semantics ? 1 : 0));
}

void airpore::get_data_contour(const std::string& path, bool binary) {
    check(fdtd_write_contour(h_, path.c_str(), binary ? 1 : 0));
}

}  // namespace b200
