// Host side of the B200 FDTD time-marching path: builds one device-resident
// domain from the reference's setup files and drives the time loop.
//
// Setup restates, in host FP64, the reference's per-frame geometry:
// calculation_2D::SetMovingFrame metrics (calculation_2D.cpp:405-433),
// air::cal_PML_var (air.cpp:509-937), air::cal_hill_var (air.cpp:938-1122),
// air::SetWindProfile (air.cpp:1286-1304), the porous constants
// (porous.cpp:40-51) and the TDBC constants (calculation_2D.cpp:1012-1028,
// airpore.cpp:252-254). Only 1D profiles, 2D wind and a box mask go to the
// device; the per-node 3D Jacobian and wind arrays of the reference are not
// materialised.
#include "fdtd_solver.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <cuda_runtime.h>

#include "fdtd_kernels.hpp"

namespace fdtd {

namespace {

#define FDTD_CK(x)                                                                                   \
    do {                                                                                             \
        cudaError_t e_ = (x);                                                                        \
        if (e_ != cudaSuccess)                                                                       \
            throw SolverError{-3, std::string(#x) + ": " + cudaGetErrorString(e_)};                 \
    } while (0)

[[noreturn]] void fail(int code, const std::string& msg) { throw SolverError{code, msg}; }

// TDBC poles of the reference (calculation_2D.h:73-75)
const double kTdA[6] = {8.226223820e-01, 3.732304064e-01, 9.106232372e-02,
                        4.819445335e-02, 4.225250937e-01, 1.837970986e-01};
const double kTdR[6] = {8.681310138e-01, 1.953722814e-01, 1.108067950e-02,
                        2.566498621e-03, 1.457297589e-04, 4.648583789e-02};

struct Medium {
    int I = 0, J = 0, K = 0;
    double dx = 1, dy = 1, dz = 1;
    std::vector<double> X, Z, axY, Y;  // axY: file axis (window), Y: current frame
    std::vector<double> fx, fy, fz;    // derivative factors x_over_X*rdx etc.

    void compute_x() { fx = factor(X, dx); }
    void compute_y() { fy = factor(Y, dy); }
    void compute_z() { fz = factor(Z, dz); }
    // X_over_x = (X[i+1]-X[i-1]) * (1/dx) * 0.5; with fixed-zero cross
    // metrics x_over_X = 1/X_over_x (calculation_2D.cpp:416-433, df_over_var.cpp:5-9)
    static std::vector<double> factor(const std::vector<double>& a, double d) {
        const int n = static_cast<int>(a.size());
        std::vector<double> f(n, 0.0);
        const double rd = 1.0 / d;
        for (int q = 1; q < n - 1; ++q) {
            const double m = (a[q + 1] - a[q - 1]) * rd * 0.5;
            f[q] = rd / m;
        }
        return f;
    }
};

// SpeedProfile (air.cpp:71-253) for the methods whose parameters the
// reference initialises. Returns false for methods 3 and 6, which read
// members the reference never sets. Method 7 (extension): the surface-layer
// log law V = (u* / kappa) ln(z / z0) with u* = b, calm at and below z0.
bool wind_at(int method, double b, double y, double z, double& U, double& V, double& W, double kappa = 0.41,
             double z0 = 0.01) {
    U = V = W = 0.0;
    switch (method) {
        case 7:
            V = z > z0 ? b / kappa * std::log(z / z0) : 0.0;
            return true;
        case 1:
            V = z >= 2.8 ? b * 2.8 : (z >= 0.0 ? b * z : 0.0);
            return true;
        case 2: {
            const double Rr = std::sqrt(std::pow(y - 5.0, 2) + std::pow(z - 2.0, 2));
            double alpha;
            if (std::fabs(y - 5.0) <= 1.0e-6 && std::fabs(z - 2.0) <= 1.0e-6) alpha = 0.0;
            else if (y - 5.0 >= 0.0) alpha = std::asin((y - 5.0) / Rr);
            else alpha = std::asin((y - 5.0) / Rr) + 3.1415926;
            V = -1.0 * 2.0 / (Rr + 2.0) * std::sin(alpha);
            W = 1.0 * 2.0 / (Rr + 2.0) * std::cos(alpha);
            return true;
        }
        case 3:
        case 6:
            return false;
        case 5:
            U = b * y;
            V = b * std::log(std::fabs(z) / 0.1 + 1);
            W = b * y;
            return true;
        default:
            return true;  // 4 and any other code: no wind
    }
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn tensor_map_encoder() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        FDTD_CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) fail(-3, "cuTensorMapEncodeTiled is unavailable");
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// split [a, b) into ceil((b - a) / T) near-equal pieces
void split_even(int a, int b, int T, std::vector<std::array<int, 2>>& out) {
    const int L = b - a;
    if (L <= 0) return;
    const int n = (L + T - 1) / T;
    for (int q = 0; q < n; ++q)
        out.push_back({a + static_cast<int>(static_cast<long long>(L) * q / n),
                       a + static_cast<int>(static_cast<long long>(L) * (q + 1) / n)});
}

// consecutive segments between the sorted, de-duplicated cut points in [lo, hi]
std::vector<std::array<int, 2>> segments(std::vector<int> cuts, int lo, int hi) {
    std::vector<int> c;
    for (int x : cuts) c.push_back(std::min(std::max(x, lo), hi));
    std::sort(c.begin(), c.end());
    c.erase(std::unique(c.begin(), c.end()), c.end());
    std::vector<std::array<int, 2>> out;
    for (size_t q = 0; q + 1 < c.size(); ++q) out.push_back({c[q], c[q + 1]});
    return out;
}

template <typename T>
T* dalloc(size_t n) {
    T* p = nullptr;
    if (n == 0) n = 1;
    FDTD_CK(cudaMalloc(&p, n * sizeof(T)));
    FDTD_CK(cudaMemset(p, 0, n * sizeof(T)));
    FDTD_CK(cudaDeviceSynchronize());  // the legacy-stream memset completes before any stream work
    return p;
}

}  // namespace

class SolverImplBase {
   public:
    virtual ~SolverImplBase() = default;
    ReferenceInput in;
    virtual std::array<int, 12> dims() const = 0;
    virtual std::vector<int> set_receivers(const std::vector<double>& xyz) = 0;
    virtual int n_receivers() const = 0;
    virtual void reset(int horizon) = 0;
    virtual int advance(int nsteps, double* rec_out) = 0;
    virtual void step_pressure() = 0;
    virtual void step_velocity() = 0;
    virtual void get_field(int medium, int comp, double* out) = 0;
    virtual void set_field(int medium, int comp, const double* in) = 0;
    virtual void get_psi(double* out) = 0;
    virtual void get_ground_psi(double* out) = 0;
    virtual int get_slab(int s, int comp, double* out, int* dims) = 0;
    virtual size_t state_elems() const = 0;
    virtual void copy_state(int dir, void* host) = 0;
    virtual void save_restart(const std::string& path) = 0;
    virtual void write_contour(const std::string& path, int format) = 0;
    virtual void load_restart(const std::string& path, bool reference_semantics) = 0;
    virtual long long launch_count() const = 0;
    virtual double last_device_ms() const = 0;
    virtual void set_tiling_api(int TI, int GC, int nt, int vw, int stages) = 0;
    virtual std::array<int, 5> autotune(int nsteps) = 0;
    virtual void get_receivers(int first_step, int nsteps, double* out) = 0;
    virtual void set_wait_limit(long long polls) = 0;
    virtual void set_tile_shape_api(int kind, int TI, int TV, int GC, int ns) = 0;
    virtual std::array<int, 19> tile_shape() const = 0;
    virtual void set_block_trace(bool on) = 0;
    virtual void get_block_trace(unsigned long long* out) = 0;
};

template <typename R>
class SolverImpl final : public SolverImplBase {
   public:
    SolverImpl(const std::string& dir, int device) {
        std::string e = parse_reference_case(dir, in);
        if (!e.empty()) fail(-1, e);
        device_ = device;
        FDTD_CK(cudaSetDevice(device_));
        cudaDeviceProp prop{};
        FDTD_CK(cudaGetDeviceProperties(&prop, device_));
        if (prop.major != 10) fail(-3, "the library is compiled for sm_100a (B200) only; device is sm_" + std::to_string(prop.major) +
                                           std::to_string(prop.minor));
        validate_and_build_geometry();
        // every transfer below is ordered on this stream, so host uploads at
        // frame boundaries never overtake kernels still queued for the
        // previous frame
        FDTD_CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        FDTD_CK(cudaEventCreate(&ev0_));
        FDTD_CK(cudaEventCreate(&ev1_));
        allocate();
        FDTD_CK(cudaDeviceSynchronize());
        // FB_p_v runs as one pass per step: the tiled kernel (any row
        // width) by default; the row marching kernel where a 2-row tile of
        // it fits (one thread per 16-byte column vector, at most 256 per
        // row) is kept for the batched ensemble and as a selectable
        // alternative. FB_v_p keeps the two passes.
        const int nvec = NJP_ / kVecMax;
        fused_ = in.scheme == FB_P_V;
        // (the row marching kernel has no terrain-following form and does
        // not stage the backward neighbours of upwind advection)
        old_ok_ = fused_ && !terrain_ && !in.upwind_advection && nvec <= kMarchThreads &&
                  march_smem_bytes(make_tiling(2, 16, 1, kVecMax, 0)) <= kSmemMax;
        if (old_ok_) {  // 4-row tiles where they fit shared memory, else 2-row
            const int TI = march_smem_bytes(make_tiling(4, 16, 256 / nvec, kVecMax, 0)) <= kSmemMax ? 4 : 2;
            set_tiling(TI, 16, 256, 0, 0);
        }
        if (fused_) {
            FDTD_CK(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
            for (int k = 1; k < kKinds; ++k) {
                FDTD_CK(cudaStreamCreateWithFlags(&kstream_[k], cudaStreamNonBlocking));
                FDTD_CK(cudaEventCreateWithFlags(&ev_join_[k], cudaEventDisableTiming));
            }
            tcfg_[0] = default_tile(false);
            tcfg_[1] = default_tile(true);
            tcfg_[2] = default_tile(false);
            tcfg_[3] = default_tile(false);
            tile_on_ = true;
            build_tiles();
        }
        reset(in.time_domain);
    }

    ~SolverImpl() override {
        cudaSetDevice(device_);
        if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
        for (void* p : allocs_) cudaFree(p);
        if (d_rec_out_) cudaFree(d_rec_out_);
        if (d_tiles_) cudaFree(d_tiles_);
        if (ev_fork_) cudaEventDestroy(ev_fork_);
        for (int k = 1; k < kKinds; ++k) {
            if (ev_join_[k]) cudaEventDestroy(ev_join_[k]);
            if (kstream_[k]) cudaStreamDestroy(kstream_[k]);
        }
        if (ev0_) cudaEventDestroy(ev0_);
        if (ev1_) cudaEventDestroy(ev1_);
        if (stream_) cudaStreamDestroy(stream_);
    }

    // ----------------------------------------------------------- setup
    void validate_and_build_geometry() {
        if (in.case_no != 1) fail(-2, "north face must be rigid or PML (the reference only steps CaseNo 1)");
        if (in.scheme != FB_P_V && in.scheme != FB_V_P)
            fail(-2, "only the forward-backward schemes (1 FB_v_p, 2 FB_p_v) are implemented by the reference");
        if (in.south != BT_RIGID && in.south != BT_ABSORBING && in.south != BT_POROUS)
            fail(-2, "south face must be rigid, PML or porous ground");
        if (in.mf.lead_DJ < 2) fail(-2, "moving-frame lead_DJ must be >= 2");
        if (in.mf.Judge == 1 && (in.mf.trail_DJ < 1 || in.mf.trail_DJ > in.mf.lead_DJ))
            fail(-2, "moving frame needs 1 <= trail_DJ <= lead_DJ (the reference shift reads past the window otherwise)");
        if (in.velocity_method == 3 || in.velocity_method == 6)
            fail(-2, "wind methods 3 and 6 read uninitialised profile parameters in the reference");
        const AxisFile& A = in.air;
        mf_ = in.mf;
        int J = A.JMAX, IJK = A.IJKMAX;
        if (mf_.Judge == 1) {  // calculation_2D.cpp:58-68
            if ((IJK - mf_.JMAX) % (mf_.lead_DJ - 1) != 0) {
                const int nl = (IJK - mf_.JMAX) / (mf_.lead_DJ - 1);
                IJK = mf_.JMAX + (nl + 1) * (mf_.lead_DJ - 1);
            }
            J = mf_.JMAX;
            if (J > A.JMAX) fail(-1, "coordi_air2.dat holds fewer nodes than the moving-frame window");
        } else {
            mf_.JMAX = J;
            IJK = J;
        }
        ijkmax_ = IJK;
        air_.I = A.IMAX; air_.J = J; air_.K = A.KMAX;
        if (air_.I < 3 || air_.J < 5 || air_.K < 3) fail(-2, "air grid needs at least 3 x 5 x 3 nodes");
        air_.dx = in.dx; air_.dy = in.dy; air_.dz = in.dz;
        air_.X = A.X;
        air_.Z = A.Z;
        air_.axY.assign(A.Y.begin(), A.Y.begin() + J);
        air_.Y = air_.axY;
        air_.compute_x(); air_.compute_y(); air_.compute_z();
        porous_ = in.has_pore;
        if (porous_) {
            const AxisFile& P = in.pore_axes;
            if (P.IMAX != air_.I || (mf_.Judge == 1 ? P.JMAX < J : P.JMAX != J))
                fail(-2, "porous grid must share the air grid's I and J node counts");
            if (P.KMAX < 3) fail(-2, "porous grid needs at least 3 z nodes");
            if (static_cast<int>(in.dz / in.pdz) >= 5)
                fail(-2, "air/porous z-spacing ratio >= 5: the reference's coarse/fine coupling is disabled code");
            pore_.I = P.IMAX; pore_.J = J; pore_.K = P.KMAX;
            pore_.dx = in.pdx; pore_.dy = in.pdy; pore_.dz = in.pdz;
            pore_.X = P.X;
            pore_.Z = P.Z;
            pore_.axY.assign(P.Y.begin(), P.Y.begin() + J);
            pore_.Y = pore_.axY;
            pore_.compute_x(); pore_.compute_y(); pore_.compute_z();
        }
        NI_ = air_.I;
        NJ_ = air_.J;
        // field rows padded to 16 bytes so whole rows can move as bulk copies
        NJP_ = (NJ_ * static_cast<int>(sizeof(R)) + 15) / 16 * 16 / static_cast<int>(sizeof(R));
        Kair_ = air_.K;
        if (porous_) {
            gAir0_ = pore_.K - 1;
            gOff_ = pore_.K - 2;
            NG_ = (pore_.K - 1) + (air_.K - 1);
        } else {
            gAir0_ = 0;
            gOff_ = 0;
            NG_ = air_.K;
        }
        build_terrain();
        // device indexing of fields and PML slabs is 32-bit
        if (static_cast<double>(NG_) * NI_ * NJP_ >= 2147483647.0)
            fail(-2, "domain holds 2^31 or more nodes per field (32-bit device indexing)");
        build_pml_static();
        build_hill();
        // TDBC constants: t_bar = dt / tau (airpore.cpp:333, calculation_2D.cpp:1012-1028)
        tdbc_ = in.east == BT_TDBC;
        const double tb = in.dt / in.tau;
        double at = 0.0;
        for (int q = 0; q < 6; ++q) {
            td_e_[q] = std::exp(-1 * kTdR[q] * tb);
            td_adt_[q] = kTdA[q] * tb;
            at += kTdA[q] * tb;
        }
        td_den_ = 1.0 / (1 + at);
        build_ground();
        // wind presence (any non-zero value on frame 0)
        wind_on_ = false;
        for (int k = 0; k < Kair_ && !wind_on_; ++k)
            for (int j = 0; j < NJ_ && !wind_on_; ++j) {
                double U, V, W;
                wind_at(in.velocity_method, in.velocity_coef, air_.Y[j], wind_z(j, k), U, V, W, in.wind_kappa, in.wind_z0);
                if (U != 0.0 || V != 0.0 || W != 0.0) wind_on_ = true;
            }
    }

    // Terrain-following grid (no counterpart in the reference, whose cross
    // metrics are fixed at zero, calculation_2D.cpp:102-104): the ground
    // elevation z_g of every column, the air grid stretched vertically
    // between the ground and its flat top H, Z(j,k) = Z[k] + z_g(j)(1 -
    // Z[k]/H), the porous grid following the ground, Z(j,k) = Z[k] + z_g(j).
    // The PML profiles stay on the file axes.
    void build_terrain() {
        terrain_ = !in.terrain.empty();
        if (!terrain_) return;
        if (mf_.Judge == 1) fail(-2, "a terrain-following grid does not run with the moving frame");
        if (in.curve_judge != 0) fail(-2, "a terrain-following grid does not run with inclusions");
        if (air_.Z[0] != 0.0) fail(-2, "a terrain-following grid needs the air axis to start at Z = 0");
        if (porous_ && pore_.Z[pore_.K - 2] != 0.0)
            fail(-2, "a terrain-following grid needs the porous axis to end one node above Z = 0");
        Htop_ = air_.Z[Kair_ - 1];
        zg_.assign(in.terrain.begin(), in.terrain.begin() + NJ_);
        for (double z : zg_)
            if (!(z < Htop_) || !std::isfinite(z)) fail(-2, "terrain reaches the top of the air grid");
    }

    // impedance ground (extension, tdbc_ground.dat): the rigid south face as a
    // 6-pole TDBC with the east face's recursion (calculation_2D.cpp:986-1017)
    // and the file's poles; t_bar = dt / tau as on the east face
    void build_ground() {
        ground_ = in.ground_tdbc;
        if (!ground_) return;
        if (in.south != BT_RIGID) fail(-2, "the impedance ground replaces a rigid south face (south code 1)");
        if (in.scheme != FB_P_V) fail(-2, "the impedance ground is implemented for scheme FB_p_v");
        if (terrain_) fail(-2, "the impedance ground does not run on a terrain-following grid");
        const double tb = in.dt / in.g_tau;
        double at = 0.0;
        for (int q = 0; q < 6; ++q) {
            gc_.e[q] = std::exp(-1 * in.g_r[q] * tb);
            gc_.adt[q] = in.g_a[q] * tb;
            at += in.g_a[q] * tb;
        }
        gc_.den = 1.0 / (1 + at);
        gc_.Z = in.g_zinf;
    }

    // physical height of node (j, k) of the air (pore = false) or porous grid
    double zh(bool pore, int j, int k) const {
        const double z = pore ? pore_.Z[k] : air_.Z[k];
        if (!terrain_) return z;
        return pore ? z + zg_[j] : z + zg_[j] * (1.0 - z / Htop_);
    }
    // height above the local ground of air node (j, k): the wind profile's z
    double wind_z(int j, int k) const { return terrain_ ? zh(false, j, k) - zg_[j] : air_.Z[k]; }

    // per (g, column) z_over_Z * rdz and z_over_Y * rdz on the terrain grid,
    // from central differences of the node heights (the reference's
    // SetMovingFrame metrics, calculation_2D.cpp:416-433, with Z(j,k)):
    // z_over_Z = X_x Y_y J = 1 / Z_z, z_over_Y = -X_x Z_y J = -Z_y / (Y_y Z_z)
    void terrain_metrics(std::vector<double>& az, std::vector<double>& zy) const {
        az.assign(static_cast<size_t>(NG_) * NJP_, 0.0);
        zy.assign(static_cast<size_t>(NG_) * NJP_, 0.0);
        for (int g = 0; g < NG_; ++g) {
            const bool pore = g < gAir0_;
            const Medium& m = pore ? pore_ : air_;
            const int k = std::min(std::max(pore ? g : g - gOff_, 1), m.K - 2);
            const double rdz = 1.0 / m.dz, rdy = 1.0 / m.dy;
            for (int jj = 0; jj < NJP_; ++jj) {
                const int j = std::min(std::max(jj, 1), NJ_ - 2);
                const double Zz = (zh(pore, j, k + 1) - zh(pore, j, k - 1)) * rdz * 0.5;
                const double Zy = (zh(pore, j + 1, k) - zh(pore, j - 1, k)) * rdy * 0.5;
                const double Yy = (m.Y[j + 1] - m.Y[j - 1]) * rdy * 0.5;
                const size_t o = static_cast<size_t>(g) * NJP_ + jj;
                az[o] = rdz / Zz;
                zy[o] = -Zy / (Yy * Zz) * rdz;
            }
        }
    }

    void build_pml_static() {
        const AxisFile& A = in.air;
        jx_ = in.pml_judge_x; jy_ = in.pml_judge_y; jz_ = in.pml_judge_z;
        I1_ = A.IMAX1; I2_ = A.IMAX2; Y1_ = A.JMAX1; Y2_ = A.JMAX2; K1_ = A.KMAX1; K2_ = A.KMAX2;
        if (jx_ == 0) I1_ = I2_ = 0;
        if (jx_ == 1) I2_ = 0;
        if (jx_ == 2) I1_ = 0;
        if (jy_ == 0) Y1_ = Y2_ = 0;
        if (jy_ == 1) Y2_ = 0;
        if (jy_ == 2) Y1_ = 0;
        if (jz_ == 0) K1_ = K2_ = 0;
        if (jz_ == 1) K2_ = 0;
        if (jz_ == 2) K1_ = 0;
        auto chk = [&](int n1, int n2, int N, const char* ax) {
            if ((n1 != 0 && n1 < 2) || (n2 != 0 && n2 < 2))
                fail(-2, std::string("PML along ") + ax + " needs at least 2 nodes per layer");
            if (n1 + n2 > N - 1) fail(-2, std::string("PML layers along ") + ax + " overlap");
        };
        chk(I1_, I2_, NI_, "x");
        chk(Y1_, Y2_, NJ_, "y");
        chk(K1_, K2_, Kair_, "z");
        // widths and layer starts from the file axes (air.cpp:534-869)
        const std::vector<double>& X = air_.X;
        const std::vector<double>& Z = air_.Z;
        const std::vector<double>& aY = air_.axY;
        if (I1_) { W1_ = 1.0 / std::fabs(X[I1_ - 1] - X[0]); x1_ = X[I1_ - 1]; }
        if (I2_) { W2_ = 1.0 / std::fabs(X[NI_ - 1] - X[NI_ - I2_]); x2_ = X[NI_ - I2_]; }
        if (Y1_) { L1_ = 1.0 / std::fabs(aY[Y1_ - 1] - aY[0]); }
        if (Y2_) { L2_ = 1.0 / std::fabs(aY[NJ_ - 1] - aY[NJ_ - Y2_]); }
        if (K1_) { H1_ = 1.0 / std::fabs(Z[K1_ - 1] - Z[0]); z1_ = Z[K1_ - 1]; }
        if (K2_) { H2_ = 1.0 / std::fabs(Z[Kair_ - 1] - Z[Kair_ - K2_]); z2_ = Z[Kair_ - K2_]; }
        pml_y_time_ = (jy_ == 1 || jy_ == 3) ? in.pml_y_time : 0;
        // x and z profiles never change with the frame
        prof(NI_, I1_, I2_, in.pml_x_sigma, in.pml_x_alpha,
             [&](int i) { return (x1_ - X[i]) * W1_; }, [&](int i) { return (X[i] - x2_) * W2_; }, sx_, fx_, gx_, sdx_);
        prof(Kair_, K1_, K2_, in.pml_z_sigma, in.pml_z_alpha,
             [&](int k) { return (z1_ - Z[k]) * H1_; }, [&](int k) { return (Z[k] - z2_) * H2_; }, sz_, fz_, gz_, sdz_);
    }

    template <typename F1, typename F2>
    static void prof(int n, int n1, int n2, double smax, double alpha, F1 d1, F2 d2, std::vector<double>& s,
                     std::vector<double>& f, std::vector<double>& g, std::vector<int8_t>& side) {
        s.assign(n, 0.0); f.assign(n, 0.0); g.assign(n, 0.0); side.assign(n, 0);
        for (int q = 0; q < n; ++q) {
            double dn;
            int sd;
            if (q < n1) { dn = d1(q); sd = 1; }
            else if (n2 > 0 && q >= n - n2) { dn = d2(q); sd = 2; }
            else continue;
            const double pw = std::pow(dn, alpha);
            const double sig = smax * pw;
            const double beta = 1.0 + 25.0 * pw;
            s[q] = sig;
            f[q] = 1.0 - 1.0 / beta;
            g[q] = 1.0 / beta - 1.0;
            side[q] = static_cast<int8_t>(sd);
        }
    }

    // y profile and layer starts for frame N (air::SetWindProfile shifts PML_y1/y2, air.cpp:1289-1292)
    void build_pml_y(int N) {
        const double sh = N * (mf_.trail_DJ - 1) * air_.dy;
        const std::vector<double>& aY = air_.axY;
        if (Y1_) y1_ = (N != 0) ? aY[Y1_ - 1] + sh : aY[Y1_ - 1];
        if (Y2_) y2_ = (N != 0) ? aY[NJ_ - Y2_] + sh : aY[NJ_ - Y2_];
        const std::vector<double>& Y = air_.Y;
        prof(NJ_, Y1_, Y2_, in.pml_y_sigma, in.pml_y_alpha, [&](int j) { return (y1_ - Y[j]) * L1_; },
             [&](int j) { return (Y[j] - y2_) * L2_; }, sy_, fy_, gy_, sdy_);
    }

    // porous inclusion mask, air::cal_hill_var (air.cpp:938-1122)
    void build_hill() {
        mask_on_ = false;
        if (in.curve_judge == 0) return;
        const double* c = in.curve;
        const std::vector<double>& X = air_.X;
        const std::vector<double>& Y = air_.axY;
        const std::vector<double>& Z = air_.Z;
        int is = 0, ie = 0, js = 0, je = 0, ks = 0, ke = 0;
        for (int i = 0; i < NI_; i++) {
            if (std::fabs(X[i] - in.hill_box[0]) <= in.dx / 8.0) is = i;
            if (std::fabs(X[i] - in.hill_box[1]) <= in.dx / 8.0) { ie = i; break; }
        }
        for (int j = 0; j < NJ_; j++) {
            if (std::fabs(Y[j] - in.hill_box[2]) <= in.dy / 8.0) js = j;
            if (std::fabs(Y[j] - in.hill_box[3]) <= in.dy / 8.0) { je = j; break; }
        }
        for (int k = 0; k < Kair_; k++) {
            if (std::fabs(Z[k] - in.hill_box[4]) <= in.dz / 8.0) ks = k;
            if (std::fabs(Z[k] - in.hill_box[5]) <= in.dz / 8.0) { ke = k; break; }
        }
        if (ie < is || je < js || ke < ks) return;
        mi0_ = is; mi1_ = ie; mj0_ = js; mj1_ = je; mk0_ = ks; mk1_ = ke;
        const int ni = ie - is + 1, nj = je - js + 1, nk = ke - ks + 1;
        mask_.assign(static_cast<size_t>(ni) * nj * nk, 0);
        auto at = [&](int i, int j, int k) -> int8_t& {
            return mask_[(static_cast<size_t>(k - ks) * ni + (i - is)) * nj + (j - js)];
        };
        int ii = 0, jj = 0;
        for (int i = is; i <= ie; i++)
            for (int j = js; j <= je; j++)
                for (int k = ks; k <= ke; k++) {
                    int8_t& m = at(i, j, k);
                    double len;
                    switch (in.curve_judge) {
                        case 1:  // sphere (c, d, e), radius b
                            len = std::pow(X[i] - c[2], 2) + std::pow(Y[j] - c[3], 2) + std::pow(Z[k] - c[4], 2);
                            if (std::sqrt(len) <= c[1]) m = 1;
                            break;
                        case 2:  // axis-aligned box
                            if (X[i] >= c[0] && X[i] <= c[1] && Y[j] >= c[2] && Y[j] <= c[3] && Z[k] >= c[4] &&
                                Z[k] <= c[5])
                                m = 1;
                            break;
                        case 3:  // three rows of vertical cylinders, spacing b, radius a
                            for (jj = 0; jj < in.curve_points; jj++) {
                                len = std::pow(X[i] - c[2], 2) + std::pow(Y[j] - (c[3] + jj * c[1]), 2);
                                if (std::sqrt(len) <= c[0] && Z[k] <= c[4]) m = 1;
                                len = std::pow(X[i] - c[5], 2) + std::pow(Y[j] - (c[6] + jj * c[1]), 2);
                                if (std::sqrt(len) <= c[0] && Z[k] <= c[7]) m = 1;
                                len = std::pow(X[i] - c[8], 2) + std::pow(Y[j] - (c[9] + jj * c[1]), 2);
                                if (std::sqrt(len) <= c[0] && Z[k] <= c[10]) m = 1;
                            }
                            break;
                        case 4:  // g x f array of cylinders
                            for (ii = 0; ii < c[6]; ii++)
                                for (jj = 0; jj < c[5]; jj++) {
                                    len = std::pow(X[i] - (c[1] + ii * c[4]), 2) +
                                          std::pow(Y[j] - (c[2] + jj * c[3]), 2);
                                    if (std::sqrt(len) <= c[0]) m = 1;
                                }
                            break;
                        case 5:  // one tree at (0, 3): cone canopy (1) and trunk (2)
                            for (ii = 0; ii < 1; ii++)
                                for (jj = 0; jj < 1; jj++) {
                                    len = std::pow(X[i] - (0.0 + ii * 2.0), 2) + std::pow(Y[j] - (3.0 + jj * 2.0), 2);
                                    const double h = -25 / (9 - 1e-50) * std::sqrt(len) + 3.0;
                                    if (std::sqrt(len) <= 0.9 && Z[k] <= h && Z[k] >= 0.5) m = 1;
                                    if (std::sqrt(len) <= 0.1 && Z[k] <= 1.5) m = 2;
                                }
                            break;
                        default:
                            break;
                    }
                }
        if (in.curve_judge == 5) {
            // the reference's second trunk sweep reuses the finished loop counters (ii = jj = 1)
            for (int i = is; i <= ie; i++)
                for (int j = js; j <= je; j++)
                    for (int k = ks; k <= ke; k++) {
                        const double len =
                            std::pow(X[i] - (0.0 + ii * 2.0), 2) + std::pow(Y[j] - (3.0 + jj * 2.0), 2);
                        if (std::sqrt(len) <= 0.1 && Z[k] <= 1.5) at(i, j, k) = 2;
                    }
        }
        if (in.curve_judge < 1 || in.curve_judge > 5) return;
        mask_on_ = true;
        // mask 1 uses the canopy parameters and mask 2 the trunk's (air.cpp:966-980, 1910-1944)
        const double dt = in.dt;
        const double e1 = 1.0 / in.canopy.eff_density, e2 = 1.0 / in.trunk.eff_density;
        const double ib1 = 1.0 / (1.0 + in.canopy.resistivity * dt * e1);
        const double ib2 = 1.0 / (1.0 + in.trunk.resistivity * dt * e2);
        m1_ = {ib1 * dt * e1, ib1, dt / in.canopy.Kp / in.canopy.porosity};
        m2_ = {ib2 * dt * e2, ib2, dt / in.trunk.Kp / in.trunk.porosity};
    }

    // ------------------------------------------------------- device
    template <typename T>
    T* track(T* p) {
        allocs_.push_back(p);
        return p;
    }

    void allocate() {
        const size_t N = static_cast<size_t>(NI_) * NJP_ * NG_;
        nodes_ = N;
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 4; ++c) F_[b][c] = track(dalloc<R>(N));
        // slabs: x1 x2 y1 y2 z1 z2
        SlabDesc sd[6];
        sd[0] = {0, 0, 0, I1_ ? I1_ + 1 : 0, NJ_, Kair_};
        sd[1] = {NI_ - 1 - I2_, 0, 0, I2_ ? I2_ + 1 : 0, NJ_, Kair_};
        sd[2] = {0, 0, 0, NI_, Y1_ ? Y1_ + 1 : 0, Kair_};
        sd[3] = {0, NJ_ - 1 - Y2_, 0, NI_, Y2_ ? Y2_ + 1 : 0, Kair_};
        sd[4] = {0, 0, 0, NI_, NJ_, K1_ ? K1_ + 1 : 0};
        sd[5] = {0, 0, Kair_ - 1 - K2_, NI_, NJ_, K2_ ? K2_ + 1 : 0};
        // slab rows are padded to 16 bytes from a 16-byte-aligned column
        // origin ja <= j0, so column vectors of the marching kernel load and
        // store slab rows as whole 16-byte vectors
        const int V = static_cast<int>(16 / sizeof(R));
        for (int s = 0; s < 6; ++s) {
            sd[s].ja = sd[s].j0 / V * V;
            sd[s].jp = sd[s].nj ? (sd[s].j0 + sd[s].nj - sd[s].ja + V - 1) / V * V : 0;
            slab_[s] = sd[s];
            const size_t n = static_cast<size_t>(sd[s].ni) * sd[s].jp * sd[s].nk;
            slab_n_[s] = n;
            for (int b = 0; b < 2; ++b)
                for (int c = 0; c < 4; ++c) Q_[s][b][c] = n ? track(dalloc<R>(n)) : nullptr;
        }
        // per-column metric arrays padded to the row pitch: the marching kernel
        // reads them as 16-byte vectors
        d_axA_ = track(dalloc<R>(NI_)); d_ayA_ = track(dalloc<R>(NJP_));
        d_axP_ = track(dalloc<R>(NI_)); d_ayP_ = track(dalloc<R>(NJP_));
        d_azG_ = track(dalloc<R>(NG_));
        if (terrain_) {
            d_azT_ = track(dalloc<R>(static_cast<size_t>(NG_) * NJP_));
            d_zyT_ = track(dalloc<R>(static_cast<size_t>(NG_) * NJP_));
        }
        for (int q = 0; q < 3; ++q) {
            d_sx_[q] = track(dalloc<R>(NI_));
            d_sy_[q] = track(dalloc<R>(NJ_));
            d_sz_[q] = track(dalloc<R>(Kair_));
        }
        d_sdx_ = track(dalloc<int8_t>(NI_)); d_sdy_ = track(dalloc<int8_t>(NJ_)); d_sdz_ = track(dalloc<int8_t>(Kair_));
        d_wt_ = track(dalloc<R>(wind_on_ ? kWindTables * wind_table_words() : 1));
        d_mask_ = mask_on_ ? track(dalloc<int8_t>(mask_.size())) : nullptr;
        if (mask_on_) h2d(d_mask_, mask_.data(), mask_.size());
        const size_t P = static_cast<size_t>(NI_) * Kair_ * 6;
        d_psi_[0] = track(dalloc<double>(P)); d_psi_[1] = track(dalloc<double>(P));
        if (ground_) gc_.psi = track(dalloc<double>(ground_psi_n()));
        d_rec_node_ = track(dalloc<long long>(kMaxRec));
        d_counters_ = track(dalloc<int>(2));
        d_status_ = track(dalloc<int>(1));
        // static profiles
        upload(d_axA_, air_.fx);
        upload(d_axP_, porous_ ? pore_.fx : air_.fx);
        upload(d_sx_[0], sx_); upload(d_sx_[1], fx_); upload(d_sx_[2], gx_);
        upload(d_sz_[0], sz_); upload(d_sz_[1], fz_); upload(d_sz_[2], gz_);
        h2d(d_sdx_, sdx_.data(), NI_);
        h2d(d_sdz_, sdz_.data(), Kair_);
        std::vector<double> az(NG_, 0.0);
        for (int g = 0; g < NG_; ++g) az[g] = (g < gAir0_) ? pore_.fz[g] : air_.fz[g - gOff_];
        upload(d_azG_, az);
        if (terrain_) {
            terrain_metrics(azt_h_, zyt_h_);
            upload(d_azT_, azt_h_);
            upload(d_zyT_, zyt_h_);
        }
    }

    // mean-wind coefficient tables of the device's wind terms (Dev::wt):
    // the frame's profile at every (air k, j) with the node's metrics and
    // dt folded in, for the interior air nodes (rows k = 1..Kair-2, columns
    // j = 1..NJ-2; the rest stay 0)
    static constexpr int kWindTables = 10;
    size_t wind_table_words() const { return static_cast<size_t>(Kair_) * NJP_; }
    void upload_wind_tables(const std::vector<double>& U, const std::vector<double>& V, const std::vector<double>& Wv) {
        const size_t S = wind_table_words();
        std::vector<double> t(kWindTables * S, 0.0);
        const double dt = in.dt, gdt = in.gamma * in.dt;
        for (int k = 1; k < Kair_ - 1; ++k)
            for (int j = 1; j < NJ_ - 1; ++j) {
                const size_t q = static_cast<size_t>(k) * NJ_ + j, up = q + NJ_, dn = q - NJ_;
                const size_t gq = static_cast<size_t>(k + gOff_) * NJP_ + j;
                const double ay = air_.fy[j];
                const double az = terrain_ ? azt_h_[gq] : air_.fz[k];
                const double zy = terrain_ ? zyt_h_[gq] : 0.0;
                const double zU = U[up] - U[dn], zV = V[up] - V[dn], zW = Wv[up] - Wv[dn];
                double dUdY = ay * (U[q + 1] - U[q - 1]) * 0.5, dVdY = ay * (V[q + 1] - V[q - 1]) * 0.5,
                       dWdY = ay * (Wv[q + 1] - Wv[q - 1]) * 0.5;
                if (terrain_) {
                    dUdY += zy * zU * 0.5;
                    dVdY += zy * zV * 0.5;
                    dWdY += zy * zW * 0.5;
                }
                const double dUdZ = az * zU * 0.5, dVdZ = az * zV * 0.5, dWdZ = az * zW * 0.5;
                const size_t o = static_cast<size_t>(k) * NJP_ + j;
                t[0 * S + o] = U[q] * dt;
                t[1 * S + o] = V[q] * ay * dt;
                t[2 * S + o] = (V[q] * zy + Wv[q] * az) * dt;
                t[3 * S + o] = gdt * (dVdY + dWdZ);
                t[4 * S + o] = dUdY * dt;
                t[5 * S + o] = dUdZ * dt;
                t[6 * S + o] = dVdY * dt;
                t[7 * S + o] = dVdZ * dt;
                t[8 * S + o] = dWdY * dt;
                t[9 * S + o] = dWdZ * dt;
            }
        upload(d_wt_, t);
    }

    void upload(R* dst, const std::vector<double>& src) {
        std::vector<R> t(src.begin(), src.end());
        h2d(dst, t.data(), t.size() * sizeof(R));
    }

    // stream-ordered host -> device copy; pageable sources are staged before
    // the call returns, so the host buffer may be released right after
    void h2d(void* dst, const void* src, size_t bytes) {
        FDTD_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_));
    }
    void d2h(void* dst, const void* src, size_t bytes) {
        FDTD_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream_));
        FDTD_CK(cudaStreamSynchronize(stream_));
    }
    void zero(void* dst, size_t bytes) { FDTD_CK(cudaMemsetAsync(dst, 0, bytes, stream_)); }

    // frame-dependent data: Y, y metrics, y PML profile, wind, receivers
    void upload_frame(int N) {
        const double sh = N * (mf_.trail_DJ - 1);
        for (int j = 0; j < NJ_; ++j) air_.Y[j] = (N != 0) ? air_.axY[j] + sh * air_.dy : air_.axY[j];
        air_.compute_y();
        upload(d_ayA_, air_.fy);
        if (porous_) {
            for (int j = 0; j < NJ_; ++j) pore_.Y[j] = (N != 0) ? pore_.axY[j] + sh * pore_.dy : pore_.axY[j];
            pore_.compute_y();
            upload(d_ayP_, pore_.fy);
        } else {
            upload(d_ayP_, air_.fy);
        }
        build_pml_y(N);
        if (fused_) update_xf();
        upload(d_sy_[0], sy_); upload(d_sy_[1], fy_); upload(d_sy_[2], gy_);
        h2d(d_sdy_, sdy_.data(), NJ_);
        if (wind_on_) {
            const size_t W = static_cast<size_t>(NJ_) * Kair_;
            std::vector<double> U(W), V(W), Wv(W);
            for (int k = 0; k < Kair_; ++k)
                for (int j = 0; j < NJ_; ++j) {
                    const size_t q = static_cast<size_t>(k) * NJ_ + j;
                    wind_at(in.velocity_method, in.velocity_coef, air_.Y[j], wind_z(j, k), U[q], V[q], Wv[q], in.wind_kappa, in.wind_z0);
                }
            upload_wind_tables(U, V, Wv);
        }
        frame_N_ = N;
        upload_receivers();
    }

    void upload_receivers() {
        std::vector<long long> node(kMaxRec, -1);
        const int sh = frame_N_ * (mf_.trail_DJ - 1);
        for (size_t r = 0; r < rec_idx_.size(); ++r) {
            const int ii = rec_idx_[r][0], jj = rec_idx_[r][1], kk = rec_idx_[r][2];
            // calculation_2D::get_pressure: strict interior of the current window
            if (jj >= sh && jj < NJ_ + sh) {
                const int jl = jj - sh;
                if (jl > 0 && jl < NJ_ - 1 && ii > 0 && ii < NI_ - 1 && kk > 0 && kk < Kair_ - 1)
                    node[r] = static_cast<long long>((static_cast<size_t>(kk + gOff_) * NI_ + ii) * NJP_ + jl);
            }
        }
        h2d(d_rec_node_, node.data(), sizeof(long long) * kMaxRec);
    }

    std::vector<int> set_receivers(const std::vector<double>& xyz) override {
        const int n = static_cast<int>(xyz.size() / 3);
        if (n > kMaxRec) fail(-5, "at most 64 receivers");
        rec_idx_.assign(n, {0, 0, 0});
        std::vector<int> out(3 * n);
        const std::vector<double>& X = air_.X;
        const std::vector<double>& Y = air_.axY;
        const std::vector<double>& Z = air_.Z;
        const double Yf = Y[NJ_ - 1] - Y[0];
        for (int r = 0; r < n; ++r) {  // calculation_2D::get_position + airpore.cpp:454-457
            const double rx = xyz[3 * r], ry = xyz[3 * r + 1], rz = xyz[3 * r + 2];
            int ii = 0, jj = 0, kk = 0;
            const int N = static_cast<int>(ry / Yf + 1.0e-6);
            for (int i = 0; i < NI_; i++)
                if (rx - X[i] <= in.dx / 8.0) { ii = i; break; }
            const int NN = N * (NJ_ - 1);
            bool found_k = false;
            if (NN < ijkmax_) {
                for (int j = NN; j < ijkmax_ && j - NN < NJ_; j++)
                    if (ry - N * Yf - Y[j - NN] <= in.dy / 8.0) { jj = j; break; }
                for (int k = 0; k < Kair_; k++)
                    if (rz - (terrain_ ? zh(false, jj, k) : Z[k]) <= in.dz / 8.0) { kk = k; found_k = true; break; }
            }
            if (!found_k) ii = jj = kk = 0;
            if (ii == 0 && jj == 0 && kk == 0) ii = jj = kk = 1;
            if (ii > NI_ || jj > ijkmax_ || kk > Kair_) ii = jj = kk = 1;
            rec_idx_[r] = {ii, jj, kk};
            out[3 * r] = ii; out[3 * r + 1] = jj; out[3 * r + 2] = kk;
        }
        upload_receivers();
        realloc_rec();
        graph_dirty_ = true;  // nrec is a captured kernel argument
        return out;
    }
    int n_receivers() const override { return static_cast<int>(rec_idx_.size()); }

    void realloc_rec() {
        const size_t n = static_cast<size_t>(std::max(horizon_, 1)) * std::max<size_t>(rec_idx_.size(), 1);
        if (n > rec_cap_) {
            if (d_rec_out_) cudaFree(d_rec_out_);
            d_rec_out_ = dalloc<double>(n);
            rec_cap_ = n;
            graph_dirty_ = true;
        }
    }

    // initial condition: Gaussian pulse, calculation_2D.cpp:292-314
    void reset(int horizon) override {
        FDTD_CK(cudaSetDevice(device_));
        FDTD_CK(cudaStreamSynchronize(stream_));
        horizon_ = horizon;
        realloc_rec();
        const size_t N = nodes_;
        std::vector<R> p(N), z(N, R(0));
        const double gc = 4.0 * std::log(2.0) / std::pow(in.gauss_width, 2);
        for (int g = 0; g < NG_; ++g) {
            const bool pore = g < gAir0_;
            const Medium& m = pore ? pore_ : air_;
            const int k = pore ? g : g - gOff_;
            for (int i = 0; i < NI_; ++i)
                for (int j = 0; j < NJ_; ++j) {
                    const double x = m.X[i] - in.source[0], y = m.axY[j] - in.source[1],
                                 zz = zh(pore, j, k) - in.source[2];
                    const double rr = std::sqrt(std::pow(x, 2) + std::pow(y, 2) + std::pow(zz, 2));
                    p[(static_cast<size_t>(g) * NI_ + i) * NJP_ + j] = static_cast<R>(1.0 * std::exp(-gc * rr * rr));
                }
        }
        h2d(F_[0][3], p.data(), N * sizeof(R));
        for (int c = 0; c < 3; ++c) zero(F_[0][c], N * sizeof(R));
        for (int c = 0; c < 4; ++c) zero(F_[1][c], N * sizeof(R));
        for (int s = 0; s < 6; ++s)
            for (int b = 0; b < 2; ++b)
                for (int c = 0; c < 4; ++c)
                    if (Q_[s][b][c]) zero(Q_[s][b][c], slab_n_[s] * sizeof(R));
        const size_t P = static_cast<size_t>(NI_) * Kair_ * 6;
        zero(d_psi_[0], P * sizeof(double));
        zero(d_psi_[1], P * sizeof(double));
        if (ground_) zero(gc_.psi, ground_psi_n() * sizeof(double));
        zero(d_counters_, 2 * sizeof(int));
        zero(d_status_, sizeof(int));
        par_ = 0;
        steps_ = 0;
        mf_count_ = 0;
        temp_time_ = 0;
        n_in_frame_ = 0;
        frame_started_ = false;
        done_ = false;
        upload_frame(0);
    }

    // params of one pass at parity par
    Dev<R> params(bool pressure, int par) const {
        Dev<R> d{};
        d.NI = NI_; d.NJ = NJ_; d.NG = NG_; d.NJP = NJP_;
        d.porous = porous_; d.gAir0 = gAir0_; d.gOff = gOff_; d.Kair = Kair_;
        d.rigid_south = !porous_;
        d.tdbc = tdbc_;
        d.fbvp = in.scheme == FB_V_P;
        d.upwind = in.upwind_advection ? 1 : 0;
        const bool fbpv = in.scheme == FB_P_V;
        const int o = par, nw = 1 - par;
        if (pressure) {
            const int ub = fbpv ? o : nw;  // FB_v_p: pressure uses the new velocity
            d.u_in = F_[ub][0]; d.v_in = F_[ub][1]; d.w_in = F_[ub][2];
            d.pold = F_[o][3];
            d.p_in = F_[o][3];
            d.p_out = F_[nw][3];
        } else {
            d.u_in = F_[o][0]; d.v_in = F_[o][1]; d.w_in = F_[o][2];
            d.p_in = fbpv ? F_[nw][3] : F_[o][3];
            d.pold = F_[o][3];
            d.u_out = F_[nw][0]; d.v_out = F_[nw][1]; d.w_out = F_[nw][2];
        }
        d.axA = d_axA_; d.ayA = d_ayA_; d.axP = d_axP_; d.ayP = d_ayP_; d.azG = d_azG_;
        d.azT = terrain_ ? d_azT_ : nullptr;
        d.zyT = terrain_ ? d_zyT_ : nullptr;
        const double dt = in.dt, gP0 = in.gamma * in.P0;
        d.dt = R(dt); d.gP0dt = R(in.gamma * in.P0 * dt); d.gdt = R(in.gamma * dt);
        d.Aavdt = R(in.Aav * dt); d.Aav = R(in.Aav); d.gP0 = R(gP0);
        if (porous_) {
            const double eff = 1.0 / in.pore.eff_density;
            const double beta = in.pore.resistivity * dt * eff;
            const double ib = 1.0 / (beta + 1.0);
            d.pGama = R(dt / in.pore.Kp / in.pore.porosity);
            d.pInvB = R(ib);
            d.pIBdtEff = R(ib * dt * eff);
        }
        d.sxI = d_sx_[0]; d.fxI = d_sx_[1]; d.gxI = d_sx_[2];
        d.syJ = d_sy_[0]; d.fyJ = d_sy_[1]; d.gyJ = d_sy_[2];
        d.szK = d_sz_[0]; d.fzK = d_sz_[1]; d.gzK = d_sz_[2];
        d.sdI = d_sdx_; d.sdJ = d_sdy_; d.sdK = d_sdz_;
        d.pml_y_time = pml_y_time_;
        for (int s = 0; s < 6; ++s) {
            Slab<R>& S = d.sl[s];
            S.i0 = slab_[s].i0; S.j0 = slab_[s].j0; S.k0 = slab_[s].k0;
            S.ni = slab_n_[s] ? slab_[s].ni : 0; S.nj = slab_[s].nj; S.nk = slab_[s].nk;
            S.ja = slab_[s].ja; S.jp = slab_[s].jp;
            if (!slab_n_[s]) continue;
            // Qp: pressure pass reads old (o) writes new (nw); velocity pass reads the
            // Qp the pressure pass of this step wrote. Qu/Qv/Qw mirror that.
            const int qp_cur = pressure ? o : (fbpv ? nw : o);
            const int quvw_cur = pressure ? (fbpv ? o : nw) : o;
            for (int c = 0; c < 3; ++c) { S.rd[c] = Q_[s][quvw_cur][c]; S.wr[c] = Q_[s][nw][c]; }
            S.rd[3] = Q_[s][qp_cur][3];
            S.wr[3] = Q_[s][nw][3];
        }
        d.wt = d_wt_;
        d.wtS = static_cast<int>(wind_table_words());
        d.mask = mask_on_ ? d_mask_ : nullptr;
        d.mi0 = mi0_; d.mi1 = mi1_; d.mj0 = mj0_; d.mj1 = mj1_; d.mk0 = mk0_; d.mk1 = mk1_;
        d.m1_ibdteff = R(m1_[0]); d.m1_ib = R(m1_[1]); d.m1_gama = R(m1_[2]);
        d.m2_ibdteff = R(m2_[0]); d.m2_ib = R(m2_[1]); d.m2_gama = R(m2_[2]);
        d.psi_in = d_psi_[o];
        d.psi_out = d_psi_[nw];
        for (int q = 0; q < 6; ++q) { d.td_e[q] = td_e_[q]; d.td_adt[q] = td_adt_[q]; }
        d.td_den = td_den_;
        d.td_z = in.Z_inf;
        d.nrec = static_cast<int>(rec_idx_.size());
        d.rec_node = d_rec_node_;
        d.rec_out = d_rec_out_;
        d.rec_steps = static_cast<int>(rec_cap_ / std::max<size_t>(rec_idx_.size(), 1));
        d.counters = d_counters_;
        d.trace = trace_on_ ? d_trace_ : nullptr;
        d.status = d_status_;
        d.wait_spin = wait_spin_;
        return d;
    }

    void launch_pass(bool pressure, int par, bool first) {
        const dim3 blk(32, 8, 1);
        const dim3 grd((NJ_ + 31) / 32, (NI_ + 7) / 8, NG_);
        const Dev<R> d = params(pressure, par);
        const int code = (first ? 1 : 0) | (par << 1);
        run_two_pass<R>(pressure, wind_on_, grd, blk, stream_, d, code);
        FDTD_CK(cudaGetLastError());
        ++launches_;
    }

    // params of the fused pass at parity par: every read from the time level /
    // slab buffer of this step, every write to the other one
    Dev<R> params_fused(int par) const {
        Dev<R> d = params(true, par);
        const int o = par, nw = 1 - par;
        d.u_in = F_[o][0]; d.v_in = F_[o][1]; d.w_in = F_[o][2];
        d.pold = F_[o][3]; d.p_in = F_[o][3];
        d.u_out = F_[nw][0]; d.v_out = F_[nw][1]; d.w_out = F_[nw][2]; d.p_out = F_[nw][3];
        for (int s = 0; s < 6; ++s) {
            if (!slab_n_[s]) continue;
            for (int c = 0; c < 4; ++c) { d.sl[s].rd[c] = Q_[s][o][c]; d.sl[s].wr[c] = Q_[s][nw][c]; }
        }
        return d;
    }

    // Marching tile: TI rows x all NJ columns x GC planes per block; trows
    // thread rows of NJP / VW threads (VW consecutive columns each).
    static constexpr size_t kSmemMax = 227 * 1024;
    static constexpr int kMarchThreads = 256;  // k_march launch bound
    static constexpr int kVecMax = static_cast<int>(16 / sizeof(R));
    static constexpr int kMaxStages = 12;  // mbarriers fit the 128-byte head of shared memory

    // shared memory of a tile: mbarriers, two new-pressure slots of
    // rows_max + 1 rows, and the ring of nstage planes; a stage holds at most
    // n + 1 u rows and n + W v, w and p rows each (n = rows_max + 1 stencil
    // rows, W = 1 with wind)
    size_t march_smem_bytes(const MarchTiling& t) const {
        const size_t row = static_cast<size_t>(NJP_) * sizeof(R);
        const int W = wind_on_ ? 1 : 0;
        // staged rows of the largest block: the kernel's clamped stencil rows
        // iclo .. ichi (u one more, v w p W more), as k_march computes them
        int stage_rows = 0;
        for (int bx = 0; bx < t.nrb; ++bx) {
            const int i0 = bx * t.TI, i1 = (bx == t.nrb - 1) ? NI_ : i0 + t.TI;
            const int rlo = i0 > 0 ? i0 - 1 : 0;
            const int iclo = std::min(std::max(rlo, 1), NI_ - 2), ichi = std::min(std::max(i1 - 1, 1), NI_ - 2);
            stage_rows = std::max(stage_rows, (ichi + 2 - iclo) + 3 * (ichi + 1 + W - iclo));
        }
        return 128 + 2 * static_cast<size_t>(t.rows_max + 1) * row + static_cast<size_t>(t.nstage) * stage_rows * row;
    }

    // stages: staging-ring planes (0: the minimum; planes g-1 with wind, g and
    // g+1 are in use while the later planes are in flight)
    MarchTiling make_tiling(int TI, int GC, int trows, int VW, int stages) const {
        MarchTiling t{};
        t.TI = std::max(2, std::min(TI, NI_));
        t.nrb = std::max(1, NI_ / t.TI);
        t.rows_max = (t.nrb == 1) ? NI_ : t.TI + NI_ % t.TI;
        t.GC = std::max(1, GC);
        t.nchunk = (NG_ - 2 + t.GC - 1) / t.GC;
        const int smin = 3 + (wind_on_ ? 1 : 0);
        t.nstage = stages == 0 ? smin : std::max(stages, smin);
        t.VW = VW;
        const int nvec = NJP_ / VW;
        t.trows = std::max(1, std::min({trows, kMarchThreads / nvec, t.rows_max + 1}));
        return t;
    }

    // Tile choice: TI rows, GC planes, about nt threads per block (rounded to
    // whole thread rows), vw columns per thread (0: 16 bytes; else 2 or 4
    // with vw * sizeof(R) <= 16).
    void set_tiling(int TI, int GC, int nt, int vw, int stages) {
        if (stages < 0 || stages > kMaxStages) fail(-5, "ring stages must be 0..12");
        const int VW = vw == 0 ? kVecMax : vw;
        if (VW != 2 && VW != 4) fail(-5, "column vector width must be 0, 2 or 4");
        if (VW > kVecMax) fail(-2, "column vector wider than 16 bytes");
        const int nvec = NJP_ / VW;
        if (nvec > kMarchThreads) fail(-2, "one thread row would exceed the marching kernel's block size");
        const MarchTiling t = make_tiling(TI, GC, std::max(1, nt / nvec), VW, stages);
        const size_t smem = march_smem_bytes(t);
        if (smem > kSmemMax) fail(-2, "marching tile does not fit shared memory");
        // the limit is per kernel and process-wide: always the largest tile,
        // so other solvers' larger tiles keep launching
        if (smem > 48 * 1024) {
            for_march_kernels([&](const void* k) {
                FDTD_CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSmemMax)));
            });
        }
        tiling_ = t;
        fused_threads_ = t.trows * nvec;
        fused_smem_ = smem;
        graph_dirty_ = true;
        if (!sdy_.empty()) update_xf();
    }

    void update_xf() {
        const bool xf = needs_xf(tile_on_ ? kVecMax : tiling_.VW);
        if (xf != xf_) {
            xf_ = xf;
            graph_dirty_ = true;
        }
    }

    template <bool XF>
    static const void* march_kernel(int VW, bool wind) {
        return march_kernel_ptr<R>(VW, wind, XF);
    }

    template <typename F>
    static void for_march_kernels(F f) {
        for (int VW : {2, 4}) {
            if (VW > kVecMax) continue;
            for (bool w : {true, false}) {
                f(march_kernel<true>(VW, w));
                f(march_kernel<false>(VW, w));
            }
        }
    }

    // the kernel form this domain launches with column vectors of VW: XF
    // (inclusion mask, east TDBC, vectors with both y layers, an east column
    // that starts a vector) only when the domain has one of them
    bool needs_xf(int VW) const {
        if (mask_on_ || tdbc_ || (!east_scalar<R, false>() && (NJ_ - 1) % VW == 0)) return true;
        for (int jb = 0; jb < NJ_; jb += VW) {
            int c = 0;
            for (int e = 0; e < VW && jb + e < NJ_; ++e) {
                const int s = sdy_[jb + e];
                if (s) c = (c == 0 || c == s) ? s : 3;
            }
            if (c == 3) return true;
        }
        return false;
    }

    // resident blocks per SM of the marching kernel for a block shape
    int march_occupancy(int VW, int threads, size_t smem) const {
        int n = 0;
        const void* k = needs_xf(VW) ? march_kernel<true>(VW, wind_on_) : march_kernel<false>(VW, wind_on_);
        if (smem > 48 * 1024)
            FDTD_CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSmemMax)));
        FDTD_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, threads, smem));
        return n;
    }

    // one fused step at parity par on the handle's stream; tiled form: the
    // kinds other than the generic full tiles run on streams of their own,
    // forked from and joined to it, so all launches of a step share the
    // device
    void launch_fused(int par) { launch_fused_on(par, stream_); }

    // one fused step at parity par on stream s (also an ensemble's stream);
    // returns the kernels launched. Tiled: the kinds other than the generic
    // full tiles run on this domain's kind streams, forked from s and
    // joined back to it (as in launch_fused), so the kinds of one step
    // share the device inside an ensemble too.
    int launch_fused_on(int par, cudaStream_t s) {
        if (tile_on_) {
            cudaStream_t st[kKinds];
            st[0] = s;
            FDTD_CK(cudaEventRecord(ev_fork_, s));
            for (int k = 1; k < kKinds; ++k) {
                st[k] = kstream_[k];
                if (ntile_[k]) FDTD_CK(cudaStreamWaitEvent(kstream_[k], ev_fork_, 0));
            }
            const int n = launch_tiles(par, st);
            for (int k = 1; k < kKinds; ++k)
                if (ntile_[k]) {
                    FDTD_CK(cudaEventRecord(ev_join_[k], kstream_[k]));
                    FDTD_CK(cudaStreamWaitEvent(s, ev_join_[k], 0));
                }
            return n;
        }
        if (!old_ok_) fail(-2, "rows too wide for the row marching kernel");
        const Dev<R> d = params_fused(par);
        if (xf_) launch_march<true>(d, par, s);
        else launch_march<false>(d, par, s);
        FDTD_CK(cudaGetLastError());
        ++launches_;
        return 1;
    }

    int launches_per_step() const {
        const int g = ground_ ? 1 : 0;
        if (in.scheme == FB_P_V && fused_) {
            if (!tile_on_) return 1 + g;
            int n = 0;
            for (int k = 0; k < kKinds; ++k) n += ntile_[k] ? 1 : 0;
            return n + g;
        }
        return 2 + g;
    }

    template <bool XF>
    void launch_march(const Dev<R>& d, int par, cudaStream_t s) {
        const dim3 grd(tiling_.nrb, tiling_.nchunk, 1), blk(fused_threads_, 1, 1);
        run_march<R>(tiling_.VW, wind_on_, XF, grd, blk, fused_smem_, s, d, tiling_, par);
    }

    void enqueue_step(int par) {
        if (in.scheme == FB_P_V && fused_) {
            launch_fused(par);
        } else if (in.scheme == FB_P_V) {
            launch_pass(true, par, true);
            launch_pass(false, par, false);
        } else {
            launch_pass(false, par, true);
            launch_pass(true, par, false);
        }
        if (ground_) launch_ground(par);
    }

    // impedance ground after the step at parity par, on the handle's stream
    void launch_ground(int par) {
        run_ground_tdbc<R>(stream_, params_fused(par), gc_, par);
        FDTD_CK(cudaGetLastError());
        ++launches_;
    }
    size_t ground_psi_n() const { return static_cast<size_t>(6) * NI_ * NJP_; }
    bool has_ground() const { return ground_; }

    static constexpr int kGraphSteps = 16;  // even: parity pattern repeats

    void ensure_graph() {
        if (graph_exec_ && !graph_dirty_) return;
        if (graph_exec_) { cudaGraphExecDestroy(graph_exec_); graph_exec_ = nullptr; }
        cudaGraph_t g;
        const long long before = launches_;
        FDTD_CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        for (int s = 0; s < kGraphSteps; ++s) enqueue_step(s & 1);
        FDTD_CK(cudaStreamEndCapture(stream_, &g));
        launches_ = before;
        FDTD_CK(cudaGraphInstantiate(&graph_exec_, g, 0));
        cudaGraphDestroy(g);
        graph_dirty_ = false;
    }

    // n steps of the current frame, parity-aware, graphs for the bulk
    void run_steps(int n) {
        while (n > 0 && (par_ & 1)) { enqueue_step(par_); par_ ^= 1; --n; ++steps_; }
        if (n >= kGraphSteps) {
            ensure_graph();
            while (n >= kGraphSteps) {
                FDTD_CK(cudaGraphLaunch(graph_exec_, stream_));
                launches_ += static_cast<long long>(launches_per_step()) * kGraphSteps;
                n -= kGraphSteps;
                steps_ += kGraphSteps;
            }
        }
        while (n > 0) { enqueue_step(par_); par_ ^= 1; --n; ++steps_; }
    }

    // moving-frame shift of fields and the x/z PML slabs along j
    void shift_frame() {
        const int sh = mf_.trail_DJ - 1, lead = mf_.lead_DJ, tempJ = mf_.JMAX - mf_.lead_DJ;
        // fields (all media) and p's west copy: calculation_2D.cpp:458-481
        const int rows = NI_ * NG_;
        for (int c = 0; c < 4; ++c) {
            run_shift_rows<R>(stream_, F_[par_][c], rows, NJP_, sh, lead, tempJ, NJ_, c == 3 ? 1 : 0);
            FDTD_CK(cudaGetLastError());
            ++launches_;
        }
        // the impedance ground's state moves with the frame like the fields
        if (ground_) {
            run_shift_rows<double>(stream_, gc_.psi, 6 * NI_, NJP_, sh, lead, tempJ, NJ_, 0);
            FDTD_CK(cudaGetLastError());
            ++launches_;
        }
        // air::SetQMove: x1, x2, z1, z2 slabs (the y slabs are not moved), air.cpp:2522-2729
        for (int s : {0, 1, 4, 5}) {
            if (!slab_n_[s]) continue;
            const int r = slab_[s].ni * slab_[s].nk;
            for (int c = 0; c < 4; ++c) {
                run_shift_rows<R>(stream_, Q_[s][par_][c], r, slab_[s].jp, sh, lead, tempJ, NJ_, 0);
                FDTD_CK(cudaGetLastError());
                ++launches_;
            }
        }
    }

    int frame_limit() const {  // airpore.cpp:542-560
        const int JMAX = ijkmax_;
        const double dy = in.dy, c0 = in.c0, dt = in.dt;
        const int last = static_cast<int>((JMAX - mf_.JMAX) / (mf_.lead_DJ - 1) + 1.e-6);
        int lim;
        if (mf_count_ == last || JMAX == mf_.JMAX) {
            lim = horizon_ - temp_time_;
        } else if (mf_count_ == 0) {
            lim = static_cast<int>((mf_.JMAX - 1) * dy / c0 / dt * mf_.ratio);
        } else {
            lim = static_cast<int>((mf_.trail_DJ - 1) * dy / c0 / dt);
            double lt1 = 0.0, lt2 = 0.0;
            if (mf_count_ % 10 == 0) {
                lt1 = (mf_.trail_DJ - 1) * dy / c0 / dt - lim;
                lt1 = lt1 * 10.0;
            }
            if (mf_count_ % 100 == 0) {
                lt2 = (mf_.trail_DJ - 1) * dy / c0 / dt - lim;
                lt2 = lt2 * 100 - static_cast<int>(lt2 * 10) * 10;
            }
            lim = lim + static_cast<int>(lt1) + static_cast<int>(lt2);
            if (temp_time_ + lim > horizon_) lim = horizon_ - temp_time_;
        }
        return lim;
    }

    // end of a frame: next frame index, and the end of the run after the
    // last frame or at the horizon (airpore.cpp:621-624)
    void close_frame_if_full() {
        if (n_in_frame_ < mf_limit_) return;
        mf_count_ += 1;
        temp_time_ += mf_limit_;
        frame_started_ = false;
        const int last = static_cast<int>((ijkmax_ - mf_.JMAX) / (mf_.lead_DJ - 1) + 1.e-6);
        if (!(mf_count_ <= last && temp_time_ < horizon_ && mf_.Judge == 1)) done_ = true;
    }

    int advance(int nsteps, double* rec_out) override {
        FDTD_CK(cudaSetDevice(device_));
        const int start = steps_;
        if (trace_on_) clear_block_trace();
        FDTD_CK(cudaEventRecord(ev0_, stream_));
        int left = nsteps;
        while (left > 0 && !done_) {
            if (!frame_started_) {
                mf_limit_ = frame_limit();
                if (mf_count_ != 0) shift_frame();
                upload_frame(mf_count_);
                frame_started_ = true;
                n_in_frame_ = 0;
            }
            const int todo = std::min(left, mf_limit_ - n_in_frame_);
            if (todo > 0) run_steps(todo);
            left -= std::max(todo, 0);
            n_in_frame_ += std::max(todo, 0);
            close_frame_if_full();
        }
        FDTD_CK(cudaEventRecord(ev1_, stream_));
        FDTD_CK(cudaStreamSynchronize(stream_));
        float ms = 0.f;
        FDTD_CK(cudaEventElapsedTime(&ms, ev0_, ev1_));
        last_ms_ = ms;
        int st = 0;
        d2h(&st, d_status_, sizeof(int));
        const int taken = steps_ - start;
        if (rec_out && !rec_idx_.empty() && taken > 0) {
            d2h(rec_out, d_rec_out_ + static_cast<size_t>(start) * rec_idx_.size(),
                sizeof(double) * taken * rec_idx_.size());
        }
        check_status(st);
        return taken;
    }

    // a timed-out wait leaves the step's values meaningless, so it is
    // reported before a non-finite pressure
    void check_status(int st) const {
        if (st & 2) fail(-7, "a staged plane copy did not complete within the wait limit");
        if (st & 1) fail(-4, "pressure became non-finite");
    }

    // half steps (FB_p_v): airpore::Cal_pressure, then Cal_velocity + UpdateInitialCond
    void step_pressure() override {
        FDTD_CK(cudaSetDevice(device_));
        if (in.scheme != FB_P_V) fail(-2, "half steps are exposed for FB_p_v only");
        // the receiver buffer holds horizon_ steps: a half step past it would
        // sample into memory the handle does not own
        if (steps_ >= horizon_) fail(-6, "half step past the horizon set by reset(); call reset first");
        if (!frame_started_) {
            mf_limit_ = frame_limit();
            upload_frame(mf_count_);
            frame_started_ = true;
        }
        launch_pass(true, par_, true);
        FDTD_CK(cudaStreamSynchronize(stream_));
    }
    void step_velocity() override {
        FDTD_CK(cudaSetDevice(device_));
        if (in.scheme != FB_P_V) fail(-2, "half steps are exposed for FB_p_v only");
        launch_pass(false, par_, false);
        if (ground_) launch_ground(par_);
        par_ ^= 1;
        ++steps_;
        ++n_in_frame_;
        FDTD_CK(cudaStreamSynchronize(stream_));
    }

    // ------------------------------------------------------- read-out
    std::vector<R> fetch(const R* d, size_t n) {
        std::vector<R> h(n);
        d2h(h.data(), d, n * sizeof(R));
        return h;
    }

    void medium_dims(int medium, int& I, int& J, int& K, int& g0) const {
        I = NI_; J = NJ_;
        if (medium == 0) { K = Kair_; g0 = gOff_; }
        else if (porous_) { K = pore_.K; g0 = 0; }
        else fail(-5, "no porous ground in this case");
    }

    // comp 0..3: p u v w at the current level; 4..7: the other ("nn") level
    const R* field_ptr(int comp) const {
        const int lvl = comp >= 4 ? 1 - par_ : par_;
        static const int map[4] = {3, 0, 1, 2};
        return F_[lvl][map[comp & 3]];
    }

    void get_field(int medium, int comp, double* out) override {
        if (comp < 0 || comp > 7) fail(-5, "comp must be 0..7");
        int I, J, K, g0;
        medium_dims(medium, I, J, K, g0);
        const std::vector<R> h = fetch(field_ptr(comp), nodes_);
        for (int i = 0; i < I; ++i)
            for (int j = 0; j < J; ++j)
                for (int k = 0; k < K; ++k)
                    out[(static_cast<size_t>(i) * J + j) * K + k] =
                        static_cast<double>(h[(static_cast<size_t>(k + g0) * NI_ + i) * NJP_ + j]);
    }

    void set_field(int medium, int comp, const double* src) override {
        if (comp < 0 || comp > 3) fail(-5, "comp must be 0..3");
        int I, J, K, g0;
        medium_dims(medium, I, J, K, g0);
        R* dptr = const_cast<R*>(field_ptr(comp));
        std::vector<R> h = fetch(dptr, nodes_);
        for (int i = 0; i < I; ++i)
            for (int j = 0; j < J; ++j)
                for (int k = 0; k < K; ++k)
                    h[(static_cast<size_t>(k + g0) * NI_ + i) * NJP_ + j] =
                        static_cast<R>(src[(static_cast<size_t>(i) * J + j) * K + k]);
        h2d(dptr, h.data(), nodes_ * sizeof(R));
        FDTD_CK(cudaStreamSynchronize(stream_));
    }

    void get_psi(double* out) override {
        d2h(out, d_psi_[par_], sizeof(double) * NI_ * Kair_ * 6);
    }

    // impedance-ground state as [i][j][6] (device layout [q][i][j])
    void get_ground_psi(double* out) override {
        if (!ground_) fail(-2, "the case has no impedance ground (tdbc_ground.dat)");
        std::vector<double> h(ground_psi_n());
        d2h(h.data(), gc_.psi, h.size() * sizeof(double));
        for (int i = 0; i < NI_; ++i)
            for (int j = 0; j < NJ_; ++j)
                for (int q = 0; q < 6; ++q)
                    out[(static_cast<size_t>(i) * NJ_ + j) * 6 + q] = h[(static_cast<size_t>(q) * NI_ + i) * NJP_ + j];
    }

    // ------------------------------------------------------- contour
    // Pressure contour of the current state, airpore::get_data_contour
    // (airpore.cpp:1014-1056) with calculation_2D::mpi_send_data and
    // operator<< (calculation_2D.cpp:1030-1190): every 4th node along each
    // axis plus the last one, X Y Z P per line with k outermost and i
    // innermost, scientific with 6 digits, Y shifted to the current frame;
    // a second zone for the porous ground. format 0 writes that Tecplot ASCII
    // file; format 1 a binary file: "FDTDCNT1", int32 zone count, then per
    // zone int32 I J K and float64 X[I], Y[J], Z[K], P[K][J][I].
    void write_contour(const std::string& path, int format) override {
        if (terrain_) fail(-2, "contour output lists one height per grid level; a terrain-following grid has none");
        FDTD_CK(cudaSetDevice(device_));
        if (format != 0 && format != 1) fail(-5, "contour format must be 0 (Tecplot ASCII) or 1 (binary)");
        struct Zone {
            std::string title;
            std::vector<double> x, y, z, p;  // p [k][j][i] over the kept nodes
        };
        auto keep = [](int n) {
            std::vector<int> idx;
            for (int q = 0; q < n; ++q)
                if (q % 4 == 0 || q == n - 1) idx.push_back(q);
            return idx;
        };
        auto zone = [&](int medium, const Medium& m, const char* title) {
            int I, J, K, g0;
            medium_dims(medium, I, J, K, g0);
            std::vector<double> f(static_cast<size_t>(I) * J * K);
            get_field(medium, 0, f.data());
            Zone z;
            z.title = title;
            const std::vector<int> ki = keep(I), kj = keep(J), kk = keep(K);
            for (int i : ki) z.x.push_back(m.X[i]);
            for (int j : kj) z.y.push_back(m.Y[j]);
            for (int k : kk) z.z.push_back(m.Z[k]);
            for (int k : kk)
                for (int j : kj)
                    for (int i : ki) z.p.push_back(f[(static_cast<size_t>(i) * J + j) * K + k]);
            return z;
        };
        std::vector<Zone> zones;
        zones.push_back(zone(0, air_, "Air Zone"));
        if (porous_) zones.push_back(zone(1, pore_, "south pore Zone"));
        std::ofstream f(path, std::ios::out | std::ios::trunc | std::ios::binary);
        if (!f) fail(-1, "cannot write contour file " + path);
        if (format == 0) {
            f.setf(std::ios::scientific, std::ios::floatfield);
            f.precision(6);
            if (!porous_) f << "VARIABLES = \"X\", \"Y\", \"Z\", \"P\"" << std::endl;
            for (const Zone& z : zones) {
                f << "ZONE T = \"" << z.title << "\",";
                f << "I=" << z.x.size() << ",J=" << z.y.size() << ",K=" << z.z.size() << ",F=POINT" << std::endl;
                size_t n = 0;
                for (double zz : z.z)
                    for (double yy : z.y)
                        for (double xx : z.x) f << xx << " " << yy << " " << zz << " " << z.p[n++] << " " << std::endl;
            }
        } else {
            f.write("FDTDCNT1", 8);
            const int32_t nz = static_cast<int32_t>(zones.size());
            f.write(reinterpret_cast<const char*>(&nz), 4);
            for (const Zone& z : zones) {
                const int32_t d[3] = {static_cast<int32_t>(z.x.size()), static_cast<int32_t>(z.y.size()),
                                      static_cast<int32_t>(z.z.size())};
                f.write(reinterpret_cast<const char*>(d), sizeof d);
                for (const auto* v : {&z.x, &z.y, &z.z, &z.p})
                    f.write(reinterpret_cast<const char*>(v->data()), static_cast<std::streamsize>(v->size() * 8));
            }
        }
        if (!f) fail(-1, "writing contour file " + path + " failed");
    }

    // ------------------------------------------------------- restart
    // File layout of one rank of the reference (airpore::Save_restart /
    // save_restartfile, airpore.cpp:664-796; calculation_2D::save_restart_cal,
    // calculation_2D.cpp:497-520; air::save_restart_air, air.cpp:1305-1379):
    //   "size rank index"
    //   air u v w p per node [i][j][k]
    //   air wind U V W per node [i][j][k], then the PML integrals Qu Qv Qw Qp
    //   per node: x1, x2 as [i][j][k], y1, y2 as [j][k][i], z1, z2 as [k][i][j]
    //   porous u v w p per node [i][j][k] (porous south face only)
    // each block on one line, scientific, sign shown, 10 digits. This library
    // appends one block the reference does not write (its reader stops
    // before it): "B200 1 MF_count temp_time n_in_frame frame_started" and
    // the TDBC state Psi [i][air k][6], so that a restart is exact for the
    // moving frame and the TDBC too.
    void save_restart(const std::string& path) override {
        FDTD_CK(cudaSetDevice(device_));
        if (ground_) fail(-2, "restart files do not carry the impedance ground's state");
        std::ofstream f(path, std::ios::out | std::ios::trunc | std::ios::binary);
        if (!f) fail(-1, "cannot write restart file " + path);
        f << 1 << " " << 0 << " " << steps_ << std::endl;
        f.setf(std::ios::scientific, std::ios::floatfield);
        f.setf(std::ios::showpos);
        f.precision(10);
        auto section = [&](auto&& body) {
            f.width(18);  // the reference sets it once per block; it pads the first value only
            body();
            f << std::endl;
        };
        auto put = [&](double v) { f << v << " "; };
        const size_t na = static_cast<size_t>(NI_) * NJ_ * Kair_;
        std::vector<double> fa[4];
        for (int c = 0; c < 4; ++c) { fa[c].resize(na); get_field(0, c, fa[c].data()); }  // p u v w
        section([&] {
            for (size_t n = 0; n < na; ++n) { put(fa[1][n]); put(fa[2][n]); put(fa[3][n]); put(fa[0][n]); }
        });
        section([&] {
            for (int i = 0; i < NI_; ++i)
                for (int j = 0; j < NJ_; ++j)
                    for (int k = 0; k < Kair_; ++k) {
                        double U = 0, V = 0, W = 0;
                        if (wind_on_) wind_at(in.velocity_method, in.velocity_coef, air_.Y[j], wind_z(j, k), U, V, W, in.wind_kappa, in.wind_z0);
                        put(U); put(V); put(W);
                    }
            for (int sl = 0; sl < 6; ++sl) {
                if (!slab_n_[sl]) continue;
                const SlabDesc& S = slab_[sl];
                std::vector<double> q[4];
                int dims[3];
                for (int c = 0; c < 4; ++c) { q[c].resize(slab_n_[sl]); get_slab(sl, c, q[c].data(), dims); }
                auto node = [&](int a, int b, int c) {
                    const size_t n = (static_cast<size_t>(a) * S.nj + b) * S.nk + c;
                    put(q[0][n]); put(q[1][n]); put(q[2][n]); put(q[3][n]);
                };
                if (sl < 2) { for (int a = 0; a < S.ni; ++a) for (int b = 0; b < S.nj; ++b) for (int c = 0; c < S.nk; ++c) node(a, b, c); }
                else if (sl < 4) { for (int b = 0; b < S.nj; ++b) for (int c = 0; c < S.nk; ++c) for (int a = 0; a < S.ni; ++a) node(a, b, c); }
                else { for (int c = 0; c < S.nk; ++c) for (int a = 0; a < S.ni; ++a) for (int b = 0; b < S.nj; ++b) node(a, b, c); }
            }
        });
        if (porous_) {
            const size_t np = static_cast<size_t>(NI_) * NJ_ * pore_.K;
            std::vector<double> fp[4];
            for (int c = 0; c < 4; ++c) { fp[c].resize(np); get_field(1, c, fp[c].data()); }
            section([&] {
                for (size_t n = 0; n < np; ++n) { put(fp[1][n]); put(fp[2][n]); put(fp[3][n]); put(fp[0][n]); }
            });
        }
        f.unsetf(std::ios::showpos);
        f << "B200 1 " << mf_count_ << " " << temp_time_ << " " << n_in_frame_ << " " << (frame_started_ ? 1 : 0)
          << std::endl;
        f.setf(std::ios::showpos);
        std::vector<double> psi(static_cast<size_t>(NI_) * Kair_ * 6);
        get_psi(psi.data());
        section([&] { for (double v : psi) put(v); });
        if (!f) fail(-1, "writing restart file " + path + " failed");
    }

    // Reads a restart file of the layout above (reference files included:
    // without this library's block the TDBC state starts at zero and the run
    // continues in frame 0) and makes it the current state; the next step is
    // step `index`. reference_semantics: continue as airpore::get_output does
    // after Read_restart (airpore.cpp:499-571) -- its frame loop then starts
    // frame 0 with air::SetQMove(0), which zeroes every PML integral
    // (air.cpp:2453-2517), and the TDBC state is not in its files -- so the
    // integrals and Psi restart from zero in frame 0.
    void load_restart(const std::string& path, bool reference_semantics) override {
        FDTD_CK(cudaSetDevice(device_));
        if (ground_) fail(-2, "restart files do not carry the impedance ground's state");
        std::ifstream f(path, std::ios::in | std::ios::binary);
        if (!f) fail(-1, "cannot read restart file " + path);
        int size = 0, rank = 0, index = 0;
        f >> size >> rank >> index;
        if (!f) fail(-1, "restart file " + path + ": bad header");
        if (size != 1) fail(-2, "restart files of a multi-rank run (one file per rank) are not supported");
        if (index < 0 || index >= horizon_) fail(-6, "restart step outside the horizon set by reset()");
        auto get = [&](double& v) {
            if (!(f >> v)) fail(-1, "restart file " + path + ": truncated");
        };
        const size_t na = static_cast<size_t>(NI_) * NJ_ * Kair_;
        std::vector<double> fa[4];
        for (auto& v : fa) v.resize(na);
        for (size_t n = 0; n < na; ++n) { get(fa[1][n]); get(fa[2][n]); get(fa[3][n]); get(fa[0][n]); }
        double skip;
        for (size_t n = 0; n < 3 * na; ++n) get(skip);  // wind: recomputed from input.txt for the frame
        std::vector<double> q[6][4];
        for (int sl = 0; sl < 6; ++sl) {
            if (!slab_n_[sl]) continue;
            const SlabDesc& S = slab_[sl];
            for (auto& v : q[sl]) v.assign(static_cast<size_t>(S.ni) * S.nj * S.nk, 0.0);
            auto node = [&](int a, int b, int c) {
                const size_t n = (static_cast<size_t>(a) * S.nj + b) * S.nk + c;
                get(q[sl][0][n]); get(q[sl][1][n]); get(q[sl][2][n]); get(q[sl][3][n]);
            };
            if (sl < 2) { for (int a = 0; a < S.ni; ++a) for (int b = 0; b < S.nj; ++b) for (int c = 0; c < S.nk; ++c) node(a, b, c); }
            else if (sl < 4) { for (int b = 0; b < S.nj; ++b) for (int c = 0; c < S.nk; ++c) for (int a = 0; a < S.ni; ++a) node(a, b, c); }
            else { for (int c = 0; c < S.nk; ++c) for (int a = 0; a < S.ni; ++a) for (int b = 0; b < S.nj; ++b) node(a, b, c); }
        }
        std::vector<double> fp[4];
        if (porous_) {
            const size_t np = static_cast<size_t>(NI_) * NJ_ * pore_.K;
            for (auto& v : fp) v.resize(np);
            for (size_t n = 0; n < np; ++n) { get(fp[1][n]); get(fp[2][n]); get(fp[3][n]); get(fp[0][n]); }
        }
        int mf = 0, tt = 0, nin = index, started = 1;
        std::vector<double> psi(static_cast<size_t>(NI_) * Kair_ * 6, 0.0);
        if (reference_semantics && mf_.Judge == 1) fail(-2, "the reference's restart cannot resume a moving frame");
        std::string tag;
        if (f >> tag) {
            int version = 0;
            if (tag != "B200" || !(f >> version >> mf >> tt >> nin >> started) || version != 1)
                fail(-1, "restart file " + path + ": unknown trailing block");
            for (double& v : psi) get(v);
        } else if (mf_.Judge == 1 && !reference_semantics) {
            fail(-1, "restart file " + path + " lacks the frame count a moving-frame run needs");
        }
        if (reference_semantics) {
            mf = 0; tt = 0; nin = index; started = 1;
            std::fill(psi.begin(), psi.end(), 0.0);
            for (auto& sq : q)
                for (auto& v : sq) std::fill(v.begin(), v.end(), 0.0);
        }
        // the state becomes time level 0 of step `index`
        FDTD_CK(cudaStreamSynchronize(stream_));
        par_ = 0;
        for (int lvl = 0; lvl < 2; ++lvl)
            for (int c = 0; c < 4; ++c) zero(F_[lvl][c], nodes_ * sizeof(R));
        if (porous_)
            for (int c = 0; c < 4; ++c) set_field(1, c, fp[c].data());
        for (int c = 0; c < 4; ++c) set_field(0, c, fa[c].data());
        for (int sl = 0; sl < 6; ++sl) {
            if (!slab_n_[sl]) continue;
            const SlabDesc& S = slab_[sl];
            for (int c = 0; c < 4; ++c) {
                std::vector<R> h(slab_n_[sl], R(0));
                for (int a = 0; a < S.ni; ++a)
                    for (int b = 0; b < S.nj; ++b)
                        for (int cc = 0; cc < S.nk; ++cc)
                            h[(static_cast<size_t>(cc) * S.ni + a) * S.jp + (b + S.j0 - S.ja)] =
                                static_cast<R>(q[sl][c][(static_cast<size_t>(a) * S.nj + b) * S.nk + cc]);
                h2d(Q_[sl][0][c], h.data(), slab_n_[sl] * sizeof(R));
                zero(Q_[sl][1][c], slab_n_[sl] * sizeof(R));
            }
        }
        h2d(d_psi_[0], psi.data(), psi.size() * sizeof(double));
        zero(d_psi_[1], psi.size() * sizeof(double));
        const int counters[2] = {index, index};
        h2d(d_counters_, counters, sizeof counters);
        zero(d_status_, sizeof(int));
        steps_ = index;
        mf_count_ = mf;
        temp_time_ = tt;
        n_in_frame_ = nin;
        frame_started_ = started != 0;
        done_ = false;
        upload_frame(mf_count_);
        if (frame_started_) mf_limit_ = frame_limit();
        FDTD_CK(cudaStreamSynchronize(stream_));
    }

    int get_slab(int s, int comp, double* out, int* dims) override {
        if (s < 0 || s > 5 || comp < 0 || comp > 3) fail(-5, "slab 0..5, comp 0..3");
        if (!slab_n_[s]) { dims[0] = dims[1] = dims[2] = 0; return 0; }
        const SlabDesc& S = slab_[s];
        dims[0] = S.ni; dims[1] = S.nj; dims[2] = S.nk;
        if (out) {
            const std::vector<R> h = fetch(Q_[s][par_][comp], slab_n_[s]);
            for (int a = 0; a < S.ni; ++a)
                for (int b = 0; b < S.nj; ++b)
                    for (int c = 0; c < S.nk; ++c)
                        out[(static_cast<size_t>(a) * S.nj + b) * S.nk + c] = static_cast<double>(
                            h[(static_cast<size_t>(c) * S.ni + a) * S.jp + (b + S.j0 - S.ja)]);
        }
        return 1;
    }

    size_t state_elems() const override { return nodes_; }

    void copy_state(int dir, void* host) override {
        FDTD_CK(cudaSetDevice(device_));
        static const int order[4] = {0, 1, 2, 3};  // u v w p
        char* h = static_cast<char*>(host);
        const size_t bytes = nodes_ * sizeof(R);
        for (int c : order) {
            if (dir == 0)
                FDTD_CK(cudaMemcpyAsync(h + c * bytes, F_[par_][c], bytes, cudaMemcpyDeviceToHost, stream_));
            else
                FDTD_CK(cudaMemcpyAsync(F_[par_][c], h + c * bytes, bytes, cudaMemcpyHostToDevice, stream_));
        }
        FDTD_CK(cudaStreamSynchronize(stream_));
    }

    std::array<int, 12> dims() const override {
        return {NI_, NJ_, Kair_, porous_ ? 1 : 0, porous_ ? pore_.I : 0, porous_ ? pore_.J : 0,
                porous_ ? pore_.K : 0, NG_, in.time_domain, static_cast<int>(sizeof(R) == 4),
                in.scheme == FB_V_P ? 1 : 0, steps_};
    }
    long long launch_count() const override { return launches_; }

    void set_tiling_api(int TI, int GC, int nt, int vw, int stages) override {
        FDTD_CK(cudaSetDevice(device_));
        if (!fused_) fail(-2, "tiling applies to the fused FB_p_v pass only");
        if (terrain_) fail(-2, "the row marching kernel has no terrain-following form");
        if (in.upwind_advection) fail(-2, "the row marching kernel has no upwind-advection form");
        if (!old_ok_) fail(-2, "rows too wide for the row marching kernel");
        set_tiling(TI, GC, nt, vw, stages);
        tile_on_ = false;  // the row marching kernel runs from now on
        if (!sdy_.empty()) update_xf();
        graph_dirty_ = true;
    }

    // ------------------------------------------------- tiled kernel
    // kind 0: full tiles (PML, faces, TDBC, inclusions); 1: lean tiles
    // fill: a generic or PML / face kind halves its plane chunk (down to 2
    // planes) while it has fewer than fill / 2 tiles per SM (0: never)
    struct TileCfg {
        int TI, TV, GC, ns;
        int fill = 4;
    };

    // shapes measured best on a 3.7 M-node porous-ground domain (B200)
    static TileCfg default_tile(bool lean) {
        if (sizeof(R) == 4) return lean ? TileCfg{16, 8, 8, 3} : TileCfg{8, 16, 8, 3};
        return lean ? TileCfg{8, 16, 32, 4} : TileCfg{8, 16, 16, 3};
    }

    TileGeo tile_geo(int TI, int TV, int ns) const {
        const int W = wind_on_ ? 1 : 0;
        TileGeo g{};
        g.TI = TI;
        g.TV = TV;
        // upwind wind advection keeps plane g-1 until the next barrier: one more stage
        g.ns = (wind_on_ && in.upwind_advection) ? std::max(ns, 4) : ns;
        g.srows = TI + 2 + W;
        g.svec = TV + 2 + W;
        const size_t bb = (static_cast<size_t>(g.srows) * g.svec * kVecMax * sizeof(R) + 127) / 128 * 128;
        g.box = static_cast<int>(bb / sizeof(R));
        g.pslot = (TI + 1) * (TV + 1) * kVecMax;
        g.ring_off = 128 + static_cast<int>((3 * static_cast<size_t>(g.pslot) * sizeof(R) + 127) / 128 * 128);
        return g;
    }
    static size_t tile_smem(const TileGeo& g) {
        return static_cast<size_t>(g.ring_off) + static_cast<size_t>(g.ns) * 4 * g.box * sizeof(R);
    }

    void check_tile(const TileCfg& c) const {
        if (c.TI < 2 || c.TV < 2 || c.GC < 1 || c.ns < 3 || c.ns > kMaxStages)
            fail(-5, "tile shape needs rows >= 2, column vectors >= 2, planes >= 1 and 3..12 ring stages");
        if ((c.TI + 1) * (c.TV + 1) > kTileMaxThreads) fail(-2, "tile needs more than 384 threads");
        const TileGeo g = tile_geo(c.TI, c.TV, c.ns);
        if (g.svec * kVecMax > 256 || g.srows > 256) fail(-2, "staged tile box exceeds 256 elements along an axis");
        if (tile_smem(g) > kSmemMax) fail(-2, "tile does not fit shared memory");
    }

    template <bool FULL, bool XF>
    static const void* tile_kernel(bool wind) {
        return tile_kernel_ptr<R>(FULL ? (XF ? 2 : 1) : 0, wind);
    }

    // Tile kinds: 0 generic full tiles (the east-face column vectors, where
    // the east extrapolation and TDBC live; every tile of a domain with
    // inclusions), 1 lean tiles (no PML storage, no face), 2 + LM tiles of
    // the PML / face kernel with layer set LM (bit 0 x, bit 1 y, bit 2 z).
    // Shape configurations: 0 full, 1 lean, 2 PML / face kinds.
    static constexpr int kKinds = 10;
    // tile configuration of a kind: 0 generic, 1 lean, 2 PML / face with at
    // most one layer, 3 PML edges and corners (two or three layers: shorter
    // grids, longer chains, tuned apart)
    static int cfg_of(int kind) {
        if (kind < 2) return kind;
        const int lm = kind - 2;
        return (lm & (lm - 1)) == 0 ? 2 : 3;
    }
    int form_of(int kind) const { return kind == 0 ? (xf_ ? 2 : 1) : kind == 1 ? 0 : kind + 1; }

    // Cuts the core planes x rows x column vectors into boxes at the PML
    // storage boundaries (x1 rows [0, I1], x2 rows [NI-1-I2, NI), y1 / y2
    // column vectors holding storage columns, z1 / z2 storage planes) and the
    // east-face vectors, classifies each box, splits it into tiles of its
    // kind's shape, orders the generic tiles heaviest first, and sizes every
    // launch. A box's layer set holds the axes whose storage its rows,
    // vectors or planes lie in; a box outside every storage region has no
    // node of a layer and no halo node of one whose pressure it reads (the
    // halo row next to an x storage region is its storage-only row, the last
    // column of the halo vector next to a y storage region is past the
    // layer, the plane below one next to a z storage region is its
    // storage-only plane). Face rows and the west face vector join the
    // storage boxes next to them, so no tile is a single face sheet where a
    // PML layer borders the face.
    void build_tiles() {
        ++tiles_gen_;
        const int V = kVecMax, nvec = NJP_ / V;
        for (int k = 0; k < 4; ++k) check_tile(tcfg_[k]);
        const int xa = I1_ ? I1_ + 1 : 0, xb = I2_ ? NI_ - 1 - I2_ : NI_;
        const int za = K1_ ? gOff_ + K1_ + 1 : 0, zb = K2_ ? gOff_ + Kair_ - 1 - K2_ : NG_;
        // the east-face vectors [ve, nvec) stay one segment: their tiles read
        // the pressure of columns NJ-2..NJ-4 from their own slots; the PML /
        // face kernel runs them unless the east face is the TDBC or its
        // column starts a vector (generic kernel)
        const int ve = nvec - 2;
        const bool east_generic = tdbc_ || (NJ_ - 1) % V == 0;
        if (sms_ == 0) FDTD_CK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_));
        const int ya = std::min(Y1_ ? (Y1_ + 1 + V - 1) / V : 0, ve);
        const int yb = std::min(Y2_ ? (NJ_ - 1 - Y2_) / V : nvec, ve);
        std::vector<int> rc{0, NI_, xa, xb}, vc{0, nvec, ya, yb}, gc{1, NG_ - 1, za, zb};
        // the east vectors join the y2 storage vectors before them when the
        // PML / face kernel runs them (one segment, tiles of >= 2 vectors)
        if (east_generic || !(yb < ve && ya <= yb)) vc.push_back(ve);
        if (xa == 0) rc.push_back(1);  // a face row with no x layer beside it: own segment
        if (xb == NI_) rc.push_back(NI_ - 2);
        if (ya == 0) vc.push_back(1);
        // the inclusion mask's box, widened by two rows, two column vectors
        // and two planes (a tile also computes the pressure of its halo row,
        // halo vector and warm-up plane), is cut out: only the tiles inside
        // it need the generic kernel's mask terms. A face row or column
        // computes at its clamped neighbour, so a box that reaches the
        // first or last interior row / vector takes the face with it.
        std::array<int, 2> mr{0, 0}, mv{0, 0}, mg{0, 0};
        if (mask_on_) {
            mr = {mi0_ - 2 <= 1 ? 0 : mi0_ - 2, mi1_ + 3 >= NI_ - 1 ? NI_ : mi1_ + 3};
            mv = {mj0_ / V - 2 <= 1 ? 0 : mj0_ / V - 2, mj1_ / V + 3 >= ve ? nvec : mj1_ / V + 3};
            mg = {std::max(gOff_ + mk0_ - 2, 1), std::min(gOff_ + mk1_ + 3, NG_ - 1)};
            rc.push_back(mr[0]); rc.push_back(mr[1]);
            vc.push_back(mv[0]); vc.push_back(mv[1]);
            gc.push_back(mg[0]); gc.push_back(mg[1]);
        }
        const auto rows = segments(rc, 0, NI_);
        const auto vecs = segments(vc, 0, nvec);
        const auto planes = segments(gc, 1, NG_ - 1);
        auto overlap = [](int a0, int a1, int b0, int b1) { return std::max(0, std::min(a1, b1) - std::max(a0, b0)); };
        std::vector<std::pair<long long, TileBox>> full;
        std::vector<TileBox> other[kKinds];
        int maxr[kKinds], maxv[kKinds];
        for (int k = 0; k < kKinds; ++k) maxr[k] = maxv[k] = 2;
        struct Box {
            std::array<int, 2> r, v, g;
        };
        std::vector<Box> boxes[kKinds];
        for (const auto& pr : planes)
            for (const auto& rr : rows)
                for (const auto& vr : vecs) {
                    const bool rx = rr[1] <= xa || rr[0] >= xb;
                    const bool vy1 = vr[1] <= ya, vy2 = vr[0] >= yb;
                    const bool gz = pr[1] <= za || pr[0] >= zb;
                    int kind;
                    const bool in_mask = mask_on_ && overlap(rr[0], rr[1], mr[0], mr[1]) > 0 &&
                                         overlap(vr[0], vr[1], mv[0], mv[1]) > 0 &&
                                         overlap(pr[0], pr[1], mg[0], mg[1]) > 0;
                    if (in_mask || (vr[1] > ve && east_generic) || (vy1 && vy2) || (vr[0] < ya && vr[1] > yb)) {
                        kind = 0;
                    } else {
                        const int lm = (rx ? kLmX : 0) | (vy1 || vy2 ? kLmY : 0) | (gz ? kLmZ : 0);
                        const bool faces = rr[0] < 1 || rr[1] > NI_ - 2 || vr[0] < 1 || vr[1] > ve;
                        kind = lm == 0 && !faces ? 1 : 2 + lm;
                    }
                    boxes[kind].push_back({rr, vr, pr});
                }
        // Plane chunks: a tile marches its planes one after another, so a
        // kind with few tiles is bound by that chain; the generic and PML /
        // face kinds halve their chunk (down to 2 planes) until they have at
        // least fill / 2 tiles per SM (two by default; the autotuner may
        // settle for fewer, longer chains, since the kinds share the device)
        int gck[kKinds];
        for (int kind = 0; kind < kKinds; ++kind) {
            const TileCfg& tc = tcfg_[cfg_of(kind)];
            auto count = [&](int gcs) {
                long long n = 0;
                for (const Box& bx : boxes[kind])
                    n += static_cast<long long>((bx.r[1] - bx.r[0] + tc.TI - 1) / tc.TI) *
                         ((bx.v[1] - bx.v[0] + tc.TV - 1) / tc.TV) * ((bx.g[1] - bx.g[0] + gcs - 1) / gcs);
                return n;
            };
            int gcs = tc.GC;
            if (kind != 1)
                while (gcs > 2 && 2 * count(gcs) < static_cast<long long>(tc.fill) * sms_) gcs = std::max(2, gcs / 2);
            gck[kind] = gcs;
        }
        for (int kind = 0; kind < kKinds; ++kind)
            for (const Box& bx : boxes[kind]) {
                const auto &rr = bx.r, &vr = bx.v, &pr = bx.g;
                {
                    const TileCfg& tc = tcfg_[cfg_of(kind)];
                    std::vector<std::array<int, 2>> rp, vp, gp;
                    split_even(rr[0], rr[1], tc.TI, rp);
                    split_even(vr[0], vr[1], tc.TV, vp);
                    split_even(pr[0], pr[1], gck[kind], gp);
                    for (const auto& a : rp)
                        for (const auto& bq : vp)
                            for (const auto& cq : gp) {
                                const TileBox t{a[0], a[1], bq[0], bq[1], cq[0], cq[1]};
                                maxr[kind] = std::max(maxr[kind], a[1] - a[0]);
                                maxv[kind] = std::max(maxv[kind], bq[1] - bq[0]);
                                if (kind != 0) {
                                    other[kind].push_back(t);
                                    continue;
                                }
                                // estimated cost: nodes with halos, times 1 + 2 per PML layer crossed
                                const int xl = overlap(t.i0, t.i1, 0, I1_) + overlap(t.i0, t.i1, NI_ - I2_, NI_) > 0;
                                const int yl = overlap(t.v0 * V, t.v1 * V, 0, Y1_) +
                                                   overlap(t.v0 * V, t.v1 * V, NJ_ - Y2_, NJ_) > 0;
                                const int zl = t.c1 > gAir0_ && (overlap(t.c0, t.c1, gOff_, gOff_ + K1_) +
                                                                     overlap(t.c0, t.c1, gOff_ + Kair_ - K2_, NG_) > 0);
                                const long long cost = static_cast<long long>(t.i1 - t.i0 + 1) * (t.v1 - t.v0 + 1) *
                                                       (t.c1 - t.c0 + 1) * (1 + 2 * (xl + yl + zl));
                                full.push_back({cost, t});
                            }
                }
            }
        std::stable_sort(full.begin(), full.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
        for (const auto& f : full) other[0].push_back(f.second);
        std::vector<TileBox> all;
        for (int k = 0; k < kKinds; ++k) {
            toff_[k] = static_cast<int>(all.size());
            ntile_[k] = static_cast<int>(other[k].size());
            all.insert(all.end(), other[k].begin(), other[k].end());
        }
        if (all.size() > tiles_cap_) {
            if (d_tiles_) cudaFree(d_tiles_);
            d_tiles_ = nullptr;
            FDTD_CK(cudaMalloc(&d_tiles_, sizeof(TileBox) * all.size()));
            tiles_cap_ = all.size();
        }
        FDTD_CK(cudaMemcpy(d_tiles_, all.data(), sizeof(TileBox) * all.size(), cudaMemcpyHostToDevice));
        bool big = false;
        for (int k = 0; k < kKinds; ++k) {
            const TileCfg& tc = tcfg_[cfg_of(k)];
            tgeo_[k] = tile_geo(std::max(2, std::min(maxr[k], tc.TI)), std::max(2, std::min(maxv[k], tc.TV)), tc.ns);
            tthr_[k] = ((tgeo_[k].TI + 1) * (tgeo_[k].TV + 1) + 31) / 32 * 32;
            tsmem_[k] = tile_smem(tgeo_[k]);
            encode_tile_maps(k);
            big = big || tsmem_[k] > 48 * 1024;
        }
        if (big) {
            for (bool w : {false, true})
                for (int f = 0; f < 3 + 8; ++f)
                    FDTD_CK(cudaFuncSetAttribute(tile_kernel_ptr<R>(f, w, terrain_), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 static_cast<int>(kSmemMax)));
        }
        if (!sdy_.empty()) update_xf();  // before the first frame upload, which sets it
        graph_dirty_ = true;
    }

    // tensor maps of the 8 field buffers for the staged box of tile kind k
    void encode_tile_maps(int k) {
        const TileGeo& g = tgeo_[k];
        const cuuint64_t dims[3] = {static_cast<cuuint64_t>(NJP_), static_cast<cuuint64_t>(NI_),
                                    static_cast<cuuint64_t>(NG_)};
        const cuuint64_t strides[2] = {static_cast<cuuint64_t>(NJP_) * sizeof(R),
                                       static_cast<cuuint64_t>(NI_) * NJP_ * sizeof(R)};
        const cuuint32_t box[3] = {static_cast<cuuint32_t>(g.svec * kVecMax), static_cast<cuuint32_t>(g.srows), 1};
        const cuuint32_t es[3] = {1, 1, 1};
        const CUtensorMapDataType dt = sizeof(R) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
        for (int lvl = 0; lvl < 2; ++lvl)
            for (int f = 0; f < 4; ++f) {
                if (reinterpret_cast<uintptr_t>(F_[lvl][f]) % 16) fail(-3, "field buffer not 16-byte aligned");
                const CUresult r = tensor_map_encoder()(&tmaps_[k][lvl].f[f], dt, 3, F_[lvl][f], dims, strides, box, es,
                                                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
                if (r != CUDA_SUCCESS) fail(-3, "tensor map encoding failed for the tiled kernel");
            }
    }

    // the launch that samples the receivers and publishes the step counter:
    // the generic kind, else the first PML / face kind present (the lean
    // kind never does)
    int book_kind() const {
        if (ntile_[0]) return 0;
        for (int k = 2; k < kKinds; ++k)
            if (ntile_[k]) return k;
        return -1;
    }

    void launch_tile_kind(int k, int par, cudaStream_t s) {
        const Dev<R> d = params_fused(par);
        const dim3 grd(static_cast<unsigned>(ntile_[k])), blk(static_cast<unsigned>(tthr_[k]));
        const int code = par | (k == book_kind() ? 2 : 0);
        run_tile<R>(form_of(k), wind_on_, terrain_, grd, blk, tsmem_[k], s, d, tmaps_[k][par], tgeo_[k],
                    d_tiles_ + toff_[k], code);
        FDTD_CK(cudaGetLastError());
        ++launches_;
    }

    // one step of the tiled kernel: kind k on streams[k] (several kinds
    // may share a stream); returns the kernels launched
    int launch_tiles(int par, const cudaStream_t* streams) {
        int n = 0;
        for (int k = 0; k < kKinds; ++k)
            if (ntile_[k]) {
                launch_tile_kind(k, par, streams[k]);
                ++n;
            }
        return n;
    }

    // tile shape of configuration 0 (full), 1 (lean) or 2 (PML / face
    // tiles): rows, column vectors and planes per tile, ring stages;
    // switches to the tiled kernel
    void set_tile_shape_api(int kind, int TI, int TV, int GC, int ns) override {
        FDTD_CK(cudaSetDevice(device_));
        if (!fused_) fail(-2, "tiling applies to the fused FB_p_v pass only");
        if (kind < 0 || kind > 2) fail(-5, "tile kind must be 0 (full), 1 (lean) or 2 (PML / face)");
        const TileCfg c{TI, TV, GC, ns};
        check_tile(c);
        FDTD_CK(cudaStreamSynchronize(stream_));
        tcfg_[kind] = c;
        if (kind == 2) tcfg_[3] = c;  // the API's PML / face shape sets the edges and corners too
        tile_on_ = true;
        build_tiles();
    }

    // per configuration 0..2: rows, vectors, planes, stages, threads (the
    // largest launch of that configuration), tiles; [18] = tiled kernel active
    std::array<int, 19> tile_shape() const override {
        std::array<int, 19> o{};
        for (int c = 0; c < 3; ++c) {
            o[6 * c + 0] = tcfg_[c].TI; o[6 * c + 1] = tcfg_[c].TV; o[6 * c + 2] = tcfg_[c].GC;
            o[6 * c + 3] = tcfg_[c].ns;
        }
        for (int k = 0; k < kKinds; ++k) {
            const int c = std::min(cfg_of(k), 2);  // PML / face: one and several layers together
            o[6 * c + 4] = std::max(o[6 * c + 4], ntile_[k] ? tthr_[k] : 0);
            o[6 * c + 5] += ntile_[k];
        }
        o[18] = tile_on_ ? 1 : 0;
        return o;
    }

    // Project autotuner for the tiled kernel: the lean tile shape, then the
    // PML / face shapes, then the full shape (the others at their current
    // shapes), twice over, since the kinds share the device step by step;
    // then the plane-chunk rule (fill) of the PML / face and full shapes;
    // each candidate is the better of two timings of nsteps steps on this
    // domain
    std::array<int, 5> autotune_tiles(int nsteps) {
        std::vector<TileCfg> cands;
        const int V = kVecMax;
        for (int TV : {16 / V * 2, 32 / V * 2, 64 / V * 2})
            for (int TI : {4, 8, 16})
                for (int GC : {8, 16, 32})
                    for (int ns : {3, 4}) {
                        const TileCfg c{TI, TV, GC, ns};
                        try {
                            check_tile(c);
                        } catch (const SolverError&) {
                            continue;
                        }
                        cands.push_back(c);
                    }
        // whole CUDA graphs of steps, as the time loop runs them
        const int nt = std::max(1, (nsteps + kGraphSteps - 1) / kGraphSteps) * kGraphSteps;
        const int saved_horizon = horizon_;
        reset(std::max(horizon_, (3 * nt + 2) * static_cast<int>(8 * cands.size() + 20) + 4));
        auto time_cfg = [&]() {
            build_tiles();
            advance(nt, nullptr);  // graph build and first touch outside the timing
            double best = 1e300;
            for (int rep = 0; rep < 2; ++rep) {
                advance(nt, nullptr);
                best = std::min(best, last_ms_);
            }
            return best;
        };
        for (int pass = 0; pass < 2; ++pass)
            for (int cfg : {1, 2, 3, 0}) {
                bool used = false;
                for (int k = 0; k < kKinds; ++k) used = used || (cfg_of(k) == cfg && ntile_[k]);
                if (!used) continue;
                TileCfg best = tcfg_[cfg];
                double best_ms = time_cfg();
                for (const TileCfg& c : cands) {
                    tcfg_[cfg] = c;
                    const double ms = time_cfg();
                    if (ms < best_ms) { best_ms = ms; best = c; }
                }
                tcfg_[cfg] = best;
                build_tiles();
            }
        for (int cfg : {2, 3, 0}) {
            bool used = false;
            for (int k = 0; k < kKinds; ++k) used = used || (cfg_of(k) == cfg && ntile_[k]);
            if (!used) continue;
            TileCfg best = tcfg_[cfg];
            double best_ms = time_cfg();
            for (int fill : {2, 1}) {
                tcfg_[cfg].fill = fill;
                const double ms = time_cfg();
                if (ms < best_ms) { best_ms = ms; best = tcfg_[cfg]; }
            }
            tcfg_[cfg] = best;
            build_tiles();
        }
        reset(saved_horizon);
        return {tcfg_[0].TI, tcfg_[0].GC, tthr_[0], kVecMax, tcfg_[0].ns};
    }

    // Project autotuner: time every candidate tile on this domain and keep the
    // fastest. Candidates: column vector width {2, 4} x rows per block
    // {2, 4, 8} x thread rows {1, 2, 4} x ring stages {minimum, +1, +2} x
    // plane chunks sized so the grid fills 1..4 whole waves of the
    // resident-block slots the occupancy calculator reports for that tile;
    // tiles that do not fit are skipped.
    std::array<int, 5> autotune(int nsteps) override {
        FDTD_CK(cudaSetDevice(device_));
        if (!fused_) fail(-2, "autotune applies to the fused FB_p_v pass only");
        if (tile_on_) return autotune_tiles(nsteps);
        cudaDeviceProp prop{};
        FDTD_CK(cudaGetDeviceProperties(&prop, device_));
        const int sms = prop.multiProcessorCount;
        const int smin = 3 + (wind_on_ ? 1 : 0);
        std::vector<std::array<int, 5>> cands;
        auto add = [&](const std::array<int, 5>& c) {
            if (std::find(cands.begin(), cands.end(), c) == cands.end()) cands.push_back(c);
        };
        for (int VW : {2, 4}) {
            if (VW > kVecMax || NJP_ / VW > kMarchThreads) continue;
            const int nvec = NJP_ / VW;
            for (int TI : {2, 4, 8})
                for (int tr : {1, 2, 4})
                    for (int extra = 0; extra <= 2; ++extra) {
                        const MarchTiling t0 = make_tiling(TI, 1, tr, VW, smin + extra);
                        const size_t smem = march_smem_bytes(t0);
                        if (t0.trows != tr || smem > kSmemMax) continue;
                        const int per_sm = march_occupancy(VW, tr * nvec, smem);
                        if (per_sm < 1) continue;
                        const int slots = per_sm * sms;
                        for (int waves = 1; waves <= 4; ++waves) {
                            const int chunks = std::max(1, (waves * slots) / t0.nrb);
                            const int GC = std::max(1, (NG_ - 2 + chunks - 1) / chunks);
                            add({TI, GC, tr * nvec, VW, smin + extra});
                        }
                    }
        }
        // whole CUDA graphs of steps, as the time loop runs them
        const int nt = std::max(1, (nsteps + kGraphSteps - 1) / kGraphSteps) * kGraphSteps;
        const int saved_horizon = horizon_;
        const int h = std::max(horizon_, 2 * nt * static_cast<int>(cands.size()) + 4);
        std::array<int, 5> best{tiling_.TI, tiling_.GC, fused_threads_, tiling_.VW, tiling_.nstage};
        double best_ms = 1e300;
        reset(h);
        for (const auto& c : cands) {
            set_tiling(c[0], c[1], c[2], c[3], c[4]);
            advance(nt, nullptr);  // graph build and first touch outside the timing
            advance(nt, nullptr);
            if (last_ms_ < best_ms) { best_ms = last_ms_; best = c; }
        }
        set_tiling(best[0], best[1], best[2], best[3], best[4]);
        reset(saved_horizon);
        return best;
    }
    double last_device_ms() const override { return last_ms_; }

    // receiver samples of steps [first_step, first_step + nsteps) already
    // taken, [nsteps][n_receivers]
    void get_receivers(int first_step, int nsteps, double* out) override {
        FDTD_CK(cudaSetDevice(device_));
        if (first_step < 0 || nsteps < 0 || first_step > steps_ || nsteps > steps_ - first_step)
            fail(-5, "receiver range outside the steps taken so far");
        if (rec_idx_.empty() || nsteps == 0) return;
        d2h(out, d_rec_out_ + static_cast<size_t>(first_step) * rec_idx_.size(),
            sizeof(double) * static_cast<size_t>(nsteps) * rec_idx_.size());
    }

    // block timeline of the tiled kernels (Dev::trace), cleared at the start
    // of every advance; off by default (one clock read per block then)
    void set_block_trace(bool on) override {
        FDTD_CK(cudaSetDevice(device_));
        FDTD_CK(cudaStreamSynchronize(stream_));
        if (on && !d_trace_) d_trace_ = track(dalloc<unsigned long long>(kTraceWords));
        trace_on_ = on;
        graph_dirty_ = true;  // the buffer is a captured kernel argument
    }
    void get_block_trace(unsigned long long* out) override {
        FDTD_CK(cudaSetDevice(device_));
        FDTD_CK(cudaStreamSynchronize(stream_));
        if (!d_trace_) fail(-5, "the block trace was never enabled");
        d2h(out, d_trace_, kTraceWords * sizeof(unsigned long long));
    }
    void clear_block_trace() {
        std::vector<unsigned long long> init(kTraceWords, 0ull);
        for (size_t q = 0; q < init.size(); q += 4) init[q] = ~0ull;
        FDTD_CK(cudaMemcpyAsync(d_trace_, init.data(), kTraceWords * sizeof(unsigned long long),
                                cudaMemcpyHostToDevice, stream_));
        FDTD_CK(cudaStreamSynchronize(stream_));
    }

    // polls a staged-copy wait of the fused pass makes before it reports a
    // timeout (0 gives up at once; < 0 restores the default)
    void set_wait_limit(long long polls) override {
        wait_spin_ = polls < 0 ? kMbarSpin : polls;
        graph_dirty_ = true;  // the limit is a captured kernel argument
    }

    // ------------------------------------------------- ensemble member
    // What a batched launch needs from this domain: the fused-pass
    // parameters of both parities, its tile and block shape.
    struct BatchView {
        Dev<R> dev[2];
        MarchTiling tile;
        int threads;
        size_t smem;
        bool wind;
        bool xf;
        bool old_ok;  // the row marching kernel (batched launches) fits
        int par;
        bool tile_on;   // the tiled kernels run the fused step
        int tiles_gen;  // tile rebuild count
    };
    bool tiled() const { return tile_on_; }
    int device() const { return device_; }
    int horizon() const { return horizon_; }
    // Readies the domain for lock-step steps taken by batched launches
    // (frame data uploaded and complete) and returns how many of n steps it
    // can take before its horizon.
    int batch_prepare(int n) {
        FDTD_CK(cudaSetDevice(device_));
        if (!fused_) fail(-2, "ensemble members need the fused FB_p_v pass");
        if (mf_.Judge == 1) fail(-2, "ensemble members cannot use the moving frame");
        if (done_) return 0;
        if (!frame_started_) {
            mf_limit_ = frame_limit();
            upload_frame(mf_count_);
            frame_started_ = true;
            n_in_frame_ = 0;
        }
        FDTD_CK(cudaStreamSynchronize(stream_));
        return std::max(0, std::min(n, mf_limit_ - n_in_frame_));
    }
    // thread blocks one fused step launches
    long long blocks_per_step() const {
        if (tile_on_) {
            long long n = 0;
            for (int k = 0; k < kKinds; ++k) n += ntile_[k];
            return n;
        }
        return static_cast<long long>(tiling_.nrb) * tiling_.nchunk;
    }
    BatchView batch_view() const {
        BatchView v{};
        v.dev[0] = params_fused(0);
        v.dev[1] = params_fused(1);
        v.tile = tiling_;
        v.threads = fused_threads_;
        v.smem = fused_smem_;
        v.wind = wind_on_;
        v.xf = old_ok_ ? needs_xf(tiling_.VW) : true;
        v.old_ok = old_ok_;
        v.par = par_;
        v.tile_on = tile_on_;
        v.tiles_gen = tiles_gen_;
        return v;
    }
    // n steps were taken by batched launches
    void batch_commit(int n, double ms) {
        if (n & 1) par_ ^= 1;
        steps_ += n;
        n_in_frame_ += n;
        last_ms_ = ms;
        close_frame_if_full();
    }
    void batch_check_status() {
        int st = 0;
        d2h(&st, d_status_, sizeof(int));
        check_status(st);
    }

   private:
    struct SlabDesc {
        int i0, j0, k0, ni, nj, nk;
        int ja = 0, jp = 0;  // 16-byte-aligned column origin and padded row pitch
    };

    int device_ = 0;
    MovingFrameCfg mf_;
    int ijkmax_ = 0;
    Medium air_, pore_;
    bool porous_ = false;
    int NI_ = 0, NJ_ = 0, NJP_ = 0, NG_ = 0, Kair_ = 0, gAir0_ = 0, gOff_ = 0;
    size_t nodes_ = 0;
    // PML
    int jx_ = 0, jy_ = 0, jz_ = 0, I1_ = 0, I2_ = 0, Y1_ = 0, Y2_ = 0, K1_ = 0, K2_ = 0, pml_y_time_ = 0;
    double W1_ = 0, W2_ = 0, L1_ = 0, L2_ = 0, H1_ = 0, H2_ = 0, x1_ = 0, x2_ = 0, y1_ = 0, y2_ = 0, z1_ = 0, z2_ = 0;
    std::vector<double> sx_, fx_, gx_, sy_, fy_, gy_, sz_, fz_, gz_;
    std::vector<int8_t> sdx_, sdy_, sdz_;
    SlabDesc slab_[6]{};
    size_t slab_n_[6]{};
    // hill
    bool mask_on_ = false;
    std::vector<int8_t> mask_;
    int mi0_ = 0, mi1_ = -1, mj0_ = 0, mj1_ = -1, mk0_ = 0, mk1_ = -1;
    std::array<double, 3> m1_{0, 0, 0}, m2_{0, 0, 0};
    // TDBC
    bool tdbc_ = false;
    double td_e_[6]{}, td_adt_[6]{}, td_den_ = 0;
    bool wind_on_ = false;
    // device
    std::vector<void*> allocs_;
    R* F_[2][4]{};
    R* Q_[6][2][4]{};
    R *d_axA_ = nullptr, *d_ayA_ = nullptr, *d_axP_ = nullptr, *d_ayP_ = nullptr, *d_azG_ = nullptr;
    // terrain-following grid: elevation per column, air top, per (g, column) factors
    bool terrain_ = false;
    bool ground_ = false;  // impedance ground (tdbc_ground.dat)
    GroundC gc_{};
    std::vector<double> zg_;
    double Htop_ = 0.0;
    R *d_azT_ = nullptr, *d_zyT_ = nullptr;
    R *d_sx_[3]{}, *d_sy_[3]{}, *d_sz_[3]{};
    int8_t *d_sdx_ = nullptr, *d_sdy_ = nullptr, *d_sdz_ = nullptr, *d_mask_ = nullptr;
    R* d_wt_ = nullptr;                  // wind coefficient tables (Dev::wt)
    std::vector<double> azt_h_, zyt_h_;  // terrain factors [g][NJP] (host copies)
    double* d_psi_[2]{};
    long long* d_rec_node_ = nullptr;
    double* d_rec_out_ = nullptr;
    size_t rec_cap_ = 0;
    int* d_counters_ = nullptr;
    int* d_status_ = nullptr;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    bool graph_dirty_ = true;
    int tiles_gen_ = 0;          // counts tile rebuilds (captured launches depend on the tiles)
    bool fused_ = false;
    bool old_ok_ = false;  // the row marching kernel fits this domain
    bool xf_ = true;  // marching kernel with the rarer features compiled in
    // tiled kernel: shape configurations (full, lean, single-layer PML) and
    // the geometry, tiles and launch of each kind
    bool tile_on_ = false;
    TileCfg tcfg_[4]{};
    static constexpr size_t kTraceWords = static_cast<size_t>(kTraceSteps) * kTraceKinds * 4;
    unsigned long long* d_trace_ = nullptr;
    bool trace_on_ = false;
    TileGeo tgeo_[kKinds]{};
    int tthr_[kKinds]{}, ntile_[kKinds]{}, toff_[kKinds]{};
    size_t tsmem_[kKinds]{};
    TileMaps tmaps_[kKinds][2]{};  // [kind][time level read]
    TileBox* d_tiles_ = nullptr;
    size_t tiles_cap_ = 0;
    cudaStream_t kstream_[kKinds]{};  // kinds 1.. (kind 0 runs on the handle's stream)
    int sms_ = 0;                     // multiprocessors of the device
    cudaEvent_t ev_fork_ = nullptr, ev_join_[kKinds]{};
    MarchTiling tiling_{};
    int fused_threads_ = 0;
    size_t fused_smem_ = 0;
    long long wait_spin_ = kMbarSpin;
    // receivers
    std::vector<std::array<int, 3>> rec_idx_;
    // time loop
    int par_ = 0, steps_ = 0, horizon_ = 0;
    int mf_count_ = 0, temp_time_ = 0, n_in_frame_ = 0, mf_limit_ = 0, frame_N_ = 0;
    bool frame_started_ = false, done_ = false;
    long long launches_ = 0;
    double last_ms_ = 0;
};

// ---------------------------------------------------------------- Solver
Solver::Solver(const std::string& case_dir, int precision, int device) : precision_(precision) {
    if (precision == 0) impl_.reset(new SolverImpl<double>(case_dir, device));
    else if (precision == 1) impl_.reset(new SolverImpl<float>(case_dir, device));
    else fail(-5, "precision must be 0 (FP64) or 1 (FP32)");
}
Solver::~Solver() = default;
const ReferenceInput& Solver::input() const { return impl_->in; }
std::array<int, 12> Solver::dims() const { return impl_->dims(); }
std::vector<int> Solver::set_receivers(const std::vector<double>& xyz) { return impl_->set_receivers(xyz); }
int Solver::n_receivers() const { return impl_->n_receivers(); }
void Solver::reset(int horizon) { impl_->reset(horizon > 0 ? horizon : impl_->in.time_domain); }
int Solver::run(int nsteps, double* rec_out) {
    impl_->reset(nsteps);
    return impl_->advance(nsteps, rec_out);
}
int Solver::advance(int nsteps, double* rec_out) { return impl_->advance(nsteps, rec_out); }
void Solver::step_pressure() { impl_->step_pressure(); }
void Solver::step_velocity() { impl_->step_velocity(); }
void Solver::get_field(int m, int c, double* out) { impl_->get_field(m, c, out); }
void Solver::set_field(int m, int c, const double* in) { impl_->set_field(m, c, in); }
void Solver::get_psi(double* out) { impl_->get_psi(out); }
void Solver::get_ground_psi(double* out) { impl_->get_ground_psi(out); }
int Solver::get_slab(int s, int c, double* out, int* dims) { return impl_->get_slab(s, c, out, dims); }
size_t Solver::state_elems() const { return impl_->state_elems(); }
void Solver::copy_state(int dir, void* host) { impl_->copy_state(dir, host); }
long long Solver::launch_count() const { return impl_->launch_count(); }
void Solver::set_tiling(int TI, int GC, int nt, int vw, int stages) { impl_->set_tiling_api(TI, GC, nt, vw, stages); }
void Solver::write_contour(const std::string& path, int format) { impl_->write_contour(path, format); }
void Solver::save_restart(const std::string& path) { impl_->save_restart(path); }
void Solver::load_restart(const std::string& path, bool reference_semantics) {
    impl_->load_restart(path, reference_semantics);
}
std::array<int, 5> Solver::autotune(int nsteps) { return impl_->autotune(nsteps); }
double Solver::last_device_ms() const { return impl_->last_device_ms(); }
void Solver::get_receivers(int first_step, int nsteps, double* out) { impl_->get_receivers(first_step, nsteps, out); }
void Solver::set_tile_shape(int kind, int TI, int TV, int GC, int ns) { impl_->set_tile_shape_api(kind, TI, TV, GC, ns); }
std::array<int, 19> Solver::tile_shape() const { return impl_->tile_shape(); }
void Solver::set_block_trace(bool on) { impl_->set_block_trace(on); }
void Solver::get_block_trace(unsigned long long* out) { impl_->get_block_trace(out); }
void Solver::set_wait_limit(long long polls) { impl_->set_wait_limit(polls); }

// ---------------------------------------------------------------- Ensemble
class EnsembleImplBase {
   public:
    virtual ~EnsembleImplBase() = default;
    virtual int advance(int nsteps) = 0;
    virtual std::array<int, 2> autotune(int nsteps) = 0;
    virtual double last_device_ms() const = 0;
    virtual long long launch_count() const = 0;
    virtual std::array<long long, 2> shape() const = 0;
    virtual void set_mode(int mode) = 0;
};

// Independent domains of one precision on one device stepped together.
// Members are grouped by kernel form (wind, column vector width) and block
// size class; every step is one launch of k_march_batch per group over the
// group's work list of (member, row block, plane chunk), heaviest blocks
// first. Groups are independent chains on their own streams, forked from
// and joined to the ensemble stream, and the time loop runs as a CUDA graph
// of kGraphSteps steps of every chain.
template <typename R>
class EnsembleImpl final : public EnsembleImplBase {
   public:
    explicit EnsembleImpl(std::vector<SolverImpl<R>*> members) : mem_(std::move(members)) {
        if (mem_.empty()) fail(-5, "an ensemble needs at least one member");
        device_ = mem_[0]->device();
        for (size_t a = 0; a < mem_.size(); ++a) {
            if (mem_[a]->device() != device_) fail(-5, "ensemble members must share one device");
            if (mem_[a]->has_ground()) fail(-5, "an ensemble member cannot have an impedance ground");
            for (size_t b = 0; b < a; ++b)
                if (mem_[a] == mem_[b]) fail(-5, "a solver appears twice in the ensemble");
        }
        FDTD_CK(cudaSetDevice(device_));
        FDTD_CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        FDTD_CK(cudaEventCreate(&ev0_));
        FDTD_CK(cudaEventCreate(&ev1_));
        FDTD_CK(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
    }
    ~EnsembleImpl() override {
        cudaSetDevice(device_);
        if (stream_) cudaStreamSynchronize(stream_);

        if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
        for (Group& g : groups_) release(g);
        for (cudaEvent_t e : mdone_) cudaEventDestroy(e);
        for (cudaStream_t s : mstreams_) cudaStreamDestroy(s);
        if (fork_) cudaEventDestroy(fork_);
        if (ev0_) cudaEventDestroy(ev0_);
        if (ev1_) cudaEventDestroy(ev1_);
        if (stream_) cudaStreamDestroy(stream_);
    }

    int advance(int nsteps) override {
        FDTD_CK(cudaSetDevice(device_));
        if (nsteps < 0) fail(-5, "negative step count");
        int n = nsteps;
        for (SolverImpl<R>* s : mem_) n = std::min(n, s->batch_prepare(nsteps));
        if (n <= 0) {
            if (nsteps > 0) fail(-6, "an ensemble member has reached its horizon; reset it");
            return 0;
        }
        plan();
        FDTD_CK(cudaEventRecord(ev0_, stream_));
        int s = 0;
        if (n >= kGraphSteps) {
            ensure_graph();
            for (; s + kGraphSteps <= n; s += kGraphSteps) {
                FDTD_CK(cudaGraphLaunch(graph_exec_, stream_));
                launches_ += static_cast<long long>(kGraphSteps) * launches_per_step();
            }
        }
        if (s < n) enqueue_steps(n - s);
        FDTD_CK(cudaEventRecord(ev1_, stream_));
        FDTD_CK(cudaStreamSynchronize(stream_));
        float ms = 0.f;
        FDTD_CK(cudaEventElapsedTime(&ms, ev0_, ev1_));
        last_ms_ = ms;
        for (SolverImpl<R>* m : mem_) m->batch_commit(n, ms);
        for (SolverImpl<R>* m : mem_) m->batch_check_status();
        return n;
    }

    // Project autotuner for the ensemble: one tile rule for every member,
    // rows per block {2, 4, 8} x plane chunk {4, 8, 16, 32} (256-thread
    // blocks of 16-byte column vectors; a member whose tile does not fit
    // shared memory keeps 2 rows), each timed over nsteps steps of the whole
    // ensemble. Every member ends reset to t = 0 with its horizon kept.
    std::array<int, 2> autotune(int nsteps) override {
        FDTD_CK(cudaSetDevice(device_));
        nsteps = std::max(nsteps, 1);
        if (mode_ == 1) {
            bool tiled = false;
            for (SolverImpl<R>* m : mem_) tiled = tiled || m->tiled();
            if (tiled) return autotune_tiles(nsteps);
        }
        std::vector<int> saved;
        for (SolverImpl<R>* m : mem_) saved.push_back(m->horizon());
        const std::array<int, 3> TIs{2, 4, 8};
        const std::array<int, 4> GCs{4, 8, 16, 32};
        const int h = (nsteps + 2) * static_cast<int>(TIs.size() * GCs.size()) + 4;
        for (SolverImpl<R>* m : mem_) m->reset(h);
        std::array<int, 2> best{0, 0};
        double best_ms = 1e300;
        for (int TI : TIs)
            for (int GC : GCs) {
                apply_tiling(TI, GC);
                advance(2);  // graph build outside the timing
                advance(nsteps);
                if (last_ms_ < best_ms) { best_ms = last_ms_; best = {TI, GC}; }
            }
        apply_tiling(best[0], best[1]);
        for (size_t i = 0; i < mem_.size(); ++i) mem_[i]->reset(saved[i]);
        return best;
    }

    // Mode 1 with tiled members: one set of tile shapes (full, lean, PML /
    // face: rows, column vectors, planes, ring stages) for every member,
    // picked from a few candidates by timing nsteps steps of the whole
    // ensemble; returns the chosen set's lean rows and planes. A candidate
    // a member cannot take (shared memory) is skipped. Every member ends
    // reset to t = 0 with its horizon kept.
    std::array<int, 2> autotune_tiles(int nsteps) {
        using C = std::array<int, 4>;
        struct Set { C full, lean, pml; };
        std::vector<Set> sets;
        if (sizeof(R) == 4)
            sets = {{{8, 16, 8, 3}, {16, 8, 8, 3}, {8, 16, 8, 3}},       {{8, 16, 8, 3}, {8, 32, 8, 4}, {8, 16, 8, 3}},
                    {{8, 16, 16, 3}, {8, 32, 16, 4}, {8, 16, 16, 3}},    {{8, 16, 16, 4}, {16, 16, 16, 4}, {8, 16, 16, 4}},
                    {{8, 8, 16, 3}, {8, 16, 32, 4}, {8, 8, 16, 3}},      {{16, 8, 16, 3}, {16, 16, 32, 4}, {16, 8, 16, 3}}};
        else
            sets = {{{8, 16, 16, 3}, {8, 16, 32, 4}, {8, 16, 16, 3}},    {{4, 16, 16, 3}, {4, 64, 16, 4}, {4, 16, 16, 3}},
                    {{8, 8, 16, 3}, {8, 32, 32, 4}, {8, 8, 16, 3}},      {{8, 16, 32, 4}, {16, 16, 32, 4}, {8, 16, 32, 4}}};
        std::vector<int> saved;
        for (SolverImpl<R>* m : mem_) saved.push_back(m->horizon());
        const int h = (nsteps + 2) * static_cast<int>(sets.size()) + 4;
        for (SolverImpl<R>* m : mem_) m->reset(h);
        int best = -1;
        double best_ms = 1e300;
        auto apply = [&](const Set& st) {
            for (SolverImpl<R>* m : mem_) {
                m->set_tile_shape_api(0, st.full[0], st.full[1], st.full[2], st.full[3]);
                m->set_tile_shape_api(1, st.lean[0], st.lean[1], st.lean[2], st.lean[3]);
                m->set_tile_shape_api(2, st.pml[0], st.pml[1], st.pml[2], st.pml[3]);
            }
        };
        for (size_t c = 0; c < sets.size(); ++c) {
            try {
                apply(sets[c]);
            } catch (const SolverError&) {
                continue;
            }
            advance(2);  // graph build outside the timing
            advance(nsteps);
            if (last_ms_ < best_ms) { best_ms = last_ms_; best = static_cast<int>(c); }
        }
        if (best < 0) fail(-2, "no tile shape set fits every member");
        apply(sets[best]);
        for (size_t i = 0; i < mem_.size(); ++i) mem_[i]->reset(saved[i]);
        return {sets[best].lean[0], sets[best].lean[2]};
    }

    double last_device_ms() const override { return last_ms_; }
    long long launch_count() const override { return launches_; }

    // 0: one k_march_batch launch per group per step; 1: every member's own
    // k_march launch (its parameters in the constant bank), members spread
    // over up to kMemberStreams streams
    void set_mode(int mode) override {
        if (mode != 0 && mode != 1) fail(-5, "ensemble mode must be 0 (batched) or 1 (per-member launches)");
        FDTD_CK(cudaSetDevice(device_));
        FDTD_CK(cudaStreamSynchronize(stream_));
        mode_ = mode;
        if (graph_exec_) { cudaGraphExecDestroy(graph_exec_); graph_exec_ = nullptr; }
        sig_.clear();
    }
    std::array<long long, 2> shape() const override {
        long long blocks = 0;
        if (mode_ == 1)
            for (const SolverImpl<R>* m : mem_) blocks += m->blocks_per_step();
        else
            for (const Group& g : groups_) blocks += static_cast<long long>(g.work.size());
        return {static_cast<long long>(groups_.size()), blocks};
    }

   private:
    static constexpr int kGraphSteps = 16;  // even: the phase pattern repeats
    static constexpr int kMemberStreams = 16;

    long long launches_per_step() const {
        return mode_ == 1 ? per_step_ : static_cast<long long>(groups_.size());
    }
    long long per_step_ = 0;  // kernels one step of mode 1 launches (counted at capture)

    struct Group {
        bool wind = false, xf = true;
        int VW = 0, threads = 0;
        size_t smem = 0;
        std::vector<int> members;  // indices into mem_
        std::vector<BatchWork> work;
        std::vector<BatchEntry<R>> entries;  // host copy, [2][members]
        BatchWork* d_work = nullptr;
        BatchEntry<R>* d_entries = nullptr;
        cudaStream_t stream = nullptr;
        cudaEvent_t done = nullptr;
    };

    // Estimated cost of block (bx, by): its cells, plus twice the cells of
    // every PML slab it updates (a slab node costs about three plain ones)
    static long long block_cost(const Dev<R>& d, const MarchTiling& tl, int bx, int by) {
        const int i0 = bx * tl.TI, i1 = (bx == tl.nrb - 1) ? d.NI : i0 + tl.TI;
        const int c0 = 1 + by * tl.GC, c1 = std::min(c0 + tl.GC, d.NG - 1);
        auto overlap = [](int a0, int a1, int b0, int b1) { return std::max(0, std::min(a1, b1) - std::max(a0, b0)); };
        const long long rows = i1 - i0, planes = c1 - c0, cols = d.NJ;
        long long slab = 0;
        for (int s = 0; s < 6; ++s) {
            const Slab<R>& S = d.sl[s];
            if (!S.ni) continue;
            slab += static_cast<long long>(overlap(i0, i1, S.i0, S.i0 + S.ni)) *
                    overlap(c0, c1, S.k0 + d.gOff, S.k0 + S.nk + d.gOff) * S.nj;
        }
        return (rows + 1) * cols * (planes + 2) + 2 * slab;
    }

    void apply_tiling(int TI, int GC) {
        for (SolverImpl<R>* m : mem_) {
            try {
                m->set_tiling_api(TI, GC, 256, 0, 0);
            } catch (const SolverError&) {
                m->set_tiling_api(2, GC, 256, 0, 0);
            }
        }
    }

    static void release(Group& g) {
        if (g.d_work) cudaFree(g.d_work);
        if (g.d_entries) cudaFree(g.d_entries);
        if (g.done) cudaEventDestroy(g.done);
        if (g.stream) cudaStreamDestroy(g.stream);
        g = Group{};
    }

    // Groups, work lists and parameter tables for the members' current
    // tiles and parities. The work lists (and so the graph) are rebuilt only
    // when a member's tile changed; the tables are refreshed every call.
    void plan() {
        std::vector<typename SolverImpl<R>::BatchView> v;
        v.reserve(mem_.size());
        for (SolverImpl<R>* m : mem_) v.push_back(m->batch_view());
        if (mode_ == 0)
            for (const auto& m : v)
                if (!m.old_ok)
                    fail(-2, "a member cannot run on the batched marching kernel (rows too wide, a "
                             "terrain-following grid or upwind advection): use mode 1");
        // block size class: 64-thread steps, so narrow (2D) members do not
        // share a launch with 256-thread blocks
        auto key_of = [&](size_t i) {
            const int cls = (v[i].threads + 63) / 64;
            return std::array<int, 4>{v[i].wind ? 1 : 0, v[i].tile.VW, cls, v[i].xf ? 1 : 0};
        };
        std::vector<std::array<int, 4>> keys;
        std::vector<int> gi(mem_.size());
        for (size_t i = 0; i < mem_.size(); ++i) {
            const auto k = key_of(i);
            auto it = std::find(keys.begin(), keys.end(), k);
            gi[i] = static_cast<int>(it - keys.begin());
            if (it == keys.end()) keys.push_back(k);
        }
        std::vector<int> sig;  // everything the captured launches depend on
        pars_.clear();
        for (size_t i = 0; i < mem_.size(); ++i) {
            const MarchTiling& tl = v[i].tile;
            sig.insert(sig.end(), {gi[i], tl.TI, tl.nrb, tl.GC, tl.nchunk, tl.rows_max, tl.nstage, tl.trows, tl.VW,
                                   v[i].threads, static_cast<int>(v[i].smem)});
            pars_.push_back(v[i].par);
            if (mode_ == 1) {  // per-member launches capture their parameters and tiles by value
                const uintptr_t r = reinterpret_cast<uintptr_t>(v[i].dev[0].rec_out);
                sig.insert(sig.end(), {v[i].par, v[i].dev[0].nrec, static_cast<int>(r), static_cast<int>(r >> 32),
                                       v[i].tile_on ? 1 : 0, v[i].tiles_gen});
            }
        }
        if (sig != sig_ || groups_.empty()) {
            if (graph_exec_) { cudaGraphExecDestroy(graph_exec_); graph_exec_ = nullptr; }
            for (Group& g : groups_) release(g);
            groups_.assign(keys.size(), Group{});
            for (size_t i = 0; i < mem_.size(); ++i) groups_[gi[i]].members.push_back(static_cast<int>(i));
            for (size_t k = 0; k < keys.size(); ++k) {
                Group& g = groups_[k];
                g.wind = keys[k][0] != 0;
                g.VW = keys[k][1];
                g.xf = keys[k][3] != 0;
                struct Costed { long long cost; BatchWork w; };
                std::vector<Costed> blocks;
                for (int a = 0; a < static_cast<int>(g.members.size()); ++a) {
                    const auto& m = v[g.members[a]];
                    g.threads = std::max(g.threads, m.threads);
                    g.smem = std::max(g.smem, m.smem);
                    const MarchTiling& tl = m.tile;
                    for (int by = 0; by < tl.nchunk; ++by)
                        for (int bx = 0; bx < tl.nrb; ++bx)
                            blocks.push_back({block_cost(m.dev[0], tl, bx, by), {a, bx, by}});
                }
                // longest blocks first: the short ones fill the last wave
                std::stable_sort(blocks.begin(), blocks.end(),
                                 [](const Costed& x, const Costed& y) { return x.cost > y.cost; });
                for (const Costed& c : blocks) g.work.push_back(c.w);
                g.threads = (g.threads + 31) / 32 * 32;
                FDTD_CK(cudaMalloc(&g.d_work, sizeof(BatchWork) * g.work.size()));
                FDTD_CK(cudaMalloc(&g.d_entries, sizeof(BatchEntry<R>) * 2 * g.members.size()));
                FDTD_CK(cudaMemcpy(g.d_work, g.work.data(), sizeof(BatchWork) * g.work.size(), cudaMemcpyHostToDevice));
                FDTD_CK(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
                FDTD_CK(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
                if (g.smem > 48 * 1024)  // process-wide per kernel: the largest tile
                    FDTD_CK(cudaFuncSetAttribute(kernel(g), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 static_cast<int>(SolverImpl<R>::kSmemMax)));
            }
            sig_ = sig;
        }
        for (Group& g : groups_) {
            const size_t nm = g.members.size();
            g.entries.resize(2 * nm);
            for (size_t a = 0; a < nm; ++a) {
                const auto& m = v[g.members[a]];
                for (int ph = 0; ph < 2; ++ph) {
                    const int par = (m.par + ph) & 1;
                    g.entries[ph * nm + a] = BatchEntry<R>{m.dev[par], m.tile, par};
                }
            }
            FDTD_CK(cudaMemcpyAsync(g.d_entries, g.entries.data(), sizeof(BatchEntry<R>) * g.entries.size(),
                                    cudaMemcpyHostToDevice, stream_));
        }
    }

    template <bool XF>
    static const void* kernel_xf(const Group& g) {
        return march_batch_kernel_ptr<R>(g.VW, g.wind, XF);
    }
    static const void* kernel(const Group& g) { return g.xf ? kernel_xf<true>(g) : kernel_xf<false>(g); }

    template <bool XF>
    void launch_xf(const Group& g, int phase) {
        const dim3 grd(static_cast<unsigned>(g.work.size())), blk(g.threads);
        const int nm = static_cast<int>(g.members.size());
        run_march_batch<R>(g.VW, g.wind, XF, grd, blk, g.smem, g.stream, g.d_work, g.d_entries, nm, phase);
    }

    void launch(const Group& g, int phase) {
        if (g.xf) launch_xf<true>(g, phase);
        else launch_xf<false>(g, phase);
        FDTD_CK(cudaGetLastError());
    }

    // n steps of every group's chain (or every member's, mode 1), forked
    // from and joined to stream_
    void enqueue_steps(int n) {
        if (mode_ == 1) {
            const int ns = static_cast<int>(std::min<size_t>(mem_.size(), kMemberStreams));
            while (static_cast<int>(mstreams_.size()) < ns) {
                cudaStream_t st;
                cudaEvent_t ev;
                FDTD_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
                FDTD_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
                mstreams_.push_back(st);
                mdone_.push_back(ev);
            }
            FDTD_CK(cudaEventRecord(fork_, stream_));
            for (int k = 0; k < ns; ++k) FDTD_CK(cudaStreamWaitEvent(mstreams_[k], fork_, 0));
            long long nl = 0;
            for (int s = 0; s < n; ++s)
                for (size_t m = 0; m < mem_.size(); ++m)
                    nl += mem_[m]->launch_fused_on((pars_[m] + s) & 1, mstreams_[m % ns]);
            for (int k = 0; k < ns; ++k) {
                FDTD_CK(cudaEventRecord(mdone_[k], mstreams_[k]));
                FDTD_CK(cudaStreamWaitEvent(stream_, mdone_[k], 0));
            }
            launches_ += nl;
            per_step_ = n > 0 ? nl / n : per_step_;
            return;
        }
        FDTD_CK(cudaEventRecord(fork_, stream_));
        for (Group& g : groups_) {
            FDTD_CK(cudaStreamWaitEvent(g.stream, fork_, 0));
            for (int s = 0; s < n; ++s) launch(g, s & 1);
            FDTD_CK(cudaEventRecord(g.done, g.stream));
            FDTD_CK(cudaStreamWaitEvent(stream_, g.done, 0));
        }
        launches_ += static_cast<long long>(n) * groups_.size();
    }

    void ensure_graph() {
        if (graph_exec_) return;
        cudaGraph_t gr;
        const long long before = launches_;
        FDTD_CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        enqueue_steps(kGraphSteps);
        FDTD_CK(cudaStreamEndCapture(stream_, &gr));
        launches_ = before;
        FDTD_CK(cudaGraphInstantiate(&graph_exec_, gr, 0));
        cudaGraphDestroy(gr);
    }

    std::vector<SolverImpl<R>*> mem_;
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr, fork_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    std::vector<Group> groups_;
    std::vector<int> sig_;
    std::vector<int> pars_;
    int mode_ = 1;  // per-member launches measured 34 % faster on the 256-member workload
    std::vector<cudaStream_t> mstreams_;
    std::vector<cudaEvent_t> mdone_;
    long long launches_ = 0;
    double last_ms_ = 0;
};

Ensemble::Ensemble(const std::vector<Solver*>& members) {
    if (members.empty()) fail(-5, "an ensemble needs at least one member");
    const int prec = members[0]->precision();
    for (Solver* s : members)
        if (!s || s->precision() != prec) fail(-5, "ensemble members must be valid solvers of one precision");
    if (prec == 0) {
        std::vector<SolverImpl<double>*> m;
        for (Solver* s : members) m.push_back(static_cast<SolverImpl<double>*>(s->impl_.get()));
        impl_.reset(new EnsembleImpl<double>(m));
    } else {
        std::vector<SolverImpl<float>*> m;
        for (Solver* s : members) m.push_back(static_cast<SolverImpl<float>*>(s->impl_.get()));
        impl_.reset(new EnsembleImpl<float>(m));
    }
}
Ensemble::~Ensemble() = default;
int Ensemble::advance(int nsteps) { return impl_->advance(nsteps); }
std::array<int, 2> Ensemble::autotune(int nsteps) { return impl_->autotune(nsteps); }
double Ensemble::last_device_ms() const { return impl_->last_device_ms(); }
long long Ensemble::launch_count() const { return impl_->launch_count(); }
std::array<long long, 2> Ensemble::shape() const { return impl_->shape(); }
void Ensemble::set_mode(int mode) { impl_->set_mode(mode); }

}  // namespace fdtd
