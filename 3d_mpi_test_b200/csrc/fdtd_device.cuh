// Device-side data model and kernels of the B200 FDTD time-marching path.
//
// One device-resident domain. Air and the porous ground layer are stacked
// in ONE column along k ("unified g axis"): the reference keeps them as two
// grids joined by a two-plane overlap copy (calculation_2D.cpp:865-985:
// air k=0 := pore K-2, pore K-1 := air k=1), which is exactly a shared
// node, so each overlap node is stored once.
//
// Layout: SoA, index ((g * NI) + i) * NJP + j, j (range / propagation axis,
// the reference's Y) contiguous, rows padded to NJP >= NJ (16-byte rows).
//
// A forward-backward step (FB_p_v, airpore.cpp:589-614) is, in the two-pass
// form of this file, two passes:
//   pressure pass  p_nn for every node, Qp slabs, receiver sampling
//   velocity pass  u,v,w_nn for every node, Qu/Qv/Qw slabs, TDBC state
// (fdtd_march.cuh holds the single-pass form.) Boundary nodes are not swept
// afterwards as in the reference (UpdateBC_*, calculation_2D.cpp:646-864);
// their final value is resolved in closed form: the BC sequence only ever
// copies from the inward neighbour, zeroes a normal component, extrapolates
// (east p) or applies the TDBC (east v), so the last face in sequence
// decides and the chain ends at an interior node whose fresh value the
// owning thread recomputes.
//
// The per-node physics (p_node, vel_node and the PML / wind / inclusion
// helpers below) is written once and shared by both forms.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fdtd {

constexpr int kMaxRec = 64;

template <typename R>
struct Slab {
    // storage range of one PML integral slab, in air node indices (k = air k)
    int i0, j0, k0, ni, nj, nk;
    int ja, jp;      // storage rows: 16-byte-aligned column origin ja <= j0, padded pitch jp
    const R* rd[4];  // u v w p  (values read this pass)
    R* wr[4];        // u v w p  (values written this pass)
    // 32-bit element index; the host rejects slabs of 2^31 elements or more
    __device__ __forceinline__ int q(int i, int j, int k) const { return ((k - k0) * ni + (i - i0)) * jp + (j - ja); }
    __device__ __forceinline__ bool holds_i(int i) const { return i >= i0 && i < i0 + ni; }
    __device__ __forceinline__ bool holds_j(int j) const { return j >= j0 && j < j0 + nj; }
    __device__ __forceinline__ bool holds_k(int k) const { return k >= k0 && k < k0 + nk; }
};

template <typename R>
struct Dev {
    int NI, NJ, NG;
    int NJP;     // row pitch of the field arrays (>= NJ; 16-byte rows)
    int porous;  // porous ground stacked below the air
    int gAir0;   // first g owned by the air medium
    int gOff;    // air k = g - gOff
    int Kair;
    int rigid_south;  // air has its own south face (rigid / absorbing)
    int tdbc;         // east face is the 6-pole TDBC
    int fbvp;         // scheme FB_v_p (velocity first)
    // advection of the velocity by the mean wind: 0 the reference's forward
    // differences (air.cpp:1476-1949), 1 backward differences (extension,
    // upwind for wind blowing toward +i/+j/+k; the WindNb neighbours are
    // then the backward ones)
    int upwind;

    // state: "in" = read, "out" = written
    const R *u_in, *v_in, *w_in, *p_in;  // old u,v,w (or new, FB_v_p pressure pass) and the p used
    const R* pold;                       // p_n (pressure pass)
    R *u_out, *v_out, *w_out, *p_out;

    // derivative factors x_over_X*rdx etc. (reference metric x scale);
    // the per-column arrays ayA / ayP are padded to NJP with zeros
    const R *axA, *ayA, *axP, *ayP, *azG;
    // terrain-following grid (null on flat ground): z_over_Z*rdz and
    // z_over_Y*rdz per (g, column), [NG][NJP]
    const R *azT, *zyT;

    // air constants
    R dt, gP0dt, gdt, Aavdt, Aav, gP0;
    // pore constants (porous.cpp:40-51)
    R pGama, pInvB, pIBdtEff;

    // PML 1D profiles: sigma, (1 - 1/beta), (1/beta - 1); side 0 none, 1 low, 2 high
    const R *sxI, *fxI, *gxI, *syJ, *fyJ, *gyJ, *szK, *fzK, *gzK;
    const int8_t *sdI, *sdJ, *sdK;
    int pml_y_time;  // y1 PML switches on once the step count reaches this
    Slab<R> sl[6];   // x1 x2 y1 y2 z1 z2 (ni == 0: absent)

    // mean-wind coefficients per (air k, j), 10 tables of wtS = Kair x NJP
    // words built by the host from the frame's wind profile (the reference
    // profiles do not depend on X) and the grid metrics, dt folded in:
    //   0 U dt, 1 V y_Y dt, 2 (V z_Y + W z_Z) dt (the z advection
    //   coefficient; z_Y = 0 off a terrain-following grid), 3 gamma dt
    //   (dV/dY + dW/dZ), 4..9 dU/dY dt, dU/dZ dt, dV/dY dt, dV/dZ dt,
    //   dW/dY dt, dW/dZ dt (central differences of the profile with the
    //   node's metrics); 0 outside the interior rows and columns
    const R* wt;
    int wtS;

    // porous inclusions in air (hill / canopy / trunk masks)
    const int8_t* mask;
    int mi0, mi1, mj0, mj1, mk0, mk1;
    R m1_ibdteff, m1_ib, m1_gama, m2_ibdteff, m2_ib, m2_gama;

    // TDBC (east face), FP64 state [i][air k][6]
    const double* psi_in;
    double* psi_out;
    double td_e[6], td_adt[6];
    double td_den, td_z;

    // receivers: p_n sampled before the step
    int nrec;
    const long long* rec_node;  // unified index or -1 (outside window / not strictly interior)
    double* rec_out;            // [step][nrec]
    int rec_steps;              // steps rec_out holds; a step at or past it records nothing
    int* counters;              // step counters (see k_pressure)
    int* status;                // bit 0: non-finite pressure seen; bit 1: staged-copy timeout
    // block timeline of the tiled kernels, or null: per step slot (step %
    // kTraceSteps) and tile kind, the earliest block start and latest block
    // end (%globaltimer, ns), the summed block durations and the blocks
    unsigned long long* trace;
    long long wait_spin;        // polls of a staged-copy wait before it reports a timeout

    __device__ __forceinline__ size_t ix(int g, int i, int j) const {
        return (static_cast<size_t>(g) * NI + i) * NJP + j;
    }
};

// ---------------------------------------------------------------- helpers
template <typename R>
__device__ __forceinline__ R ldg(const R* p) { return __ldg(p); }

template <typename R>
__device__ __forceinline__ int y_side(const Dev<R>& d, int j, bool y1_on) {
    int s = d.sdJ[j];
    if (s == 1 && !y1_on) s = 0;
    return s;
}

// PML coefficients of one axis at one node: sigma, 1 - 1/beta, 1/beta - 1
// (air.cpp:509-937 profile, beta = 1 + 25 (d/W)^alpha)
template <typename R>
struct PmlC {
    R s, f, g;
};

// N consecutive column values (N * sizeof(R) <= 16) moved as one access;
// Vec is the 16-byte column vector of the marching kernel. N = 1 is the
// node-wise form of the two-pass kernels.
template <typename R, int N>
struct alignas(sizeof(R) * N) Arr {
    R e[N];
};
template <typename R>
using Vec = Arr<R, 16 / static_cast<int>(sizeof(R))>;

template <typename R, int N>
__device__ __forceinline__ Arr<R, N> ldn(const R* p) {
    return *reinterpret_cast<const Arr<R, N>*>(p);
}
template <typename R, int N>
__device__ __forceinline__ void stn(R* p, const Arr<R, N>& v) {
    *reinterpret_cast<Arr<R, N>*>(p) = v;
}

// Compiler scheduling fence: memory accesses are not moved across it. Used
// between the x, y and z PML sections, which are mostly exclusive (a node
// lies in one layer except along edges), so hoisting every section's loads
// ahead would only raise register pressure.
__device__ __forceinline__ void sched_fence() { asm volatile("" ::: "memory"); }

// Active y PML sides of N columns are packed 2 bits per column (0 none, 1
// low, 2 high). y_common: 0 when no column is in the layer, the side when
// every active column shares it, 3 when both sides occur.
template <int N>
__device__ __forceinline__ int y_common(int ysp) {
    int c = 0;
#pragma unroll
    for (int e = 0; e < N; ++e) {
        const int s = (ysp >> (2 * e)) & 3;
        if (s) c = (c == 0 || c == s) ? s : 3;
    }
    return c;
}

// Coefficients constant over one plane g (air k = g - gOff).
template <typename R>
struct PlaneC {
    R az;
    int pore;    // porous-ground plane
    int k;       // air k
    int zs;      // active z PML side of an air plane (0 none, 1 low, 2 high)
    PmlC<R> Z;
    int inmask;  // plane crosses the inclusion box
};

template <typename R>
__device__ __forceinline__ PlaneC<R> plane_c(const Dev<R>& d, int g) {
    PlaneC<R> c;
    c.az = ldg(d.azG + g);
    c.pore = g < d.gAir0;
    c.k = g - d.gOff;
    c.zs = 0;
    c.Z = {R(0), R(0), R(0)};
    c.inmask = 0;
    if (!c.pore) {
        c.zs = d.sdK[c.k];
        if (c.zs) c.Z = {ldg(d.szK + c.k), ldg(d.fzK + c.k), ldg(d.gzK + c.k)};
        c.inmask = d.mask != nullptr && c.k >= d.mk0 && c.k <= d.mk1;
    }
    return c;
}

// Coefficients constant along one row i of a plane.
template <typename R>
struct RowC {
    R ax;
    int xs;  // active x PML side
    PmlC<R> X;
    int inmask;
};

template <typename R>
__device__ __forceinline__ RowC<R> row_c(const Dev<R>& d, const PlaneC<R>& pc, int i) {
    RowC<R> r;
    r.ax = ldg((pc.pore ? d.axP : d.axA) + i);
    r.xs = 0;
    r.X = {R(0), R(0), R(0)};
    r.inmask = pc.inmask && i >= d.mi0 && i <= d.mi1;
    if (!pc.pore) {
        r.xs = d.sdI[i];
        if (r.xs) r.X = {ldg(d.sxI + i), ldg(d.fxI + i), ldg(d.gxI + i)};
    }
    return r;
}

template <typename R>
__device__ __forceinline__ PmlC<R> pml_y(const Dev<R>& d, int ys, int j) {
    if (!ys) return {R(0), R(0), R(0)};
    return {ldg(d.syJ + j), ldg(d.fyJ + j), ldg(d.gyJ + j)};
}

// inclusion mask value at air node (i, j, k) of a row inside the box's i
// and k range: 0 air, 1 canopy, 2 trunk (air::cal_hill_var, air.cpp:938-1122)
template <typename R>
__device__ __forceinline__ int mask_at(const Dev<R>& d, int i, int j, int k) {
    if (j < d.mj0 || j > d.mj1) return 0;
    return d.mask[((k - d.mk0) * (d.mi1 - d.mi0 + 1) + (i - d.mi0)) * (d.mj1 - d.mj0 + 1) + (j - d.mj0)];
}

// element e of an N-vector as a 1-vector
template <typename R, int N>
__device__ __forceinline__ Arr<R, 1> el(const Arr<R, N>& a, int e) {
    return Arr<R, 1>{{a.e[e]}};
}

// -------------------------------------------------- terrain-following grid
// Per-column factors of one plane on a grid stretched vertically under a
// ground elevation z_g(Y) (extension of the reference's generic metric
// form, df_over_var.cpp:5-9 with the cross term z_over_Y live; use sites
// air.cpp:1476-2322, porous.cpp:58-143): z_over_Z * rdz and z_over_Y * rdz
// per (plane, column), and the v at g + 1 the cross term of div u reads.
// Without terrain (TER = false) az is the plane's 1D factor and zy is 0.
template <typename R, int N>
struct TerC {
    Arr<R, N> az, zy, vk;
};

// the factors of N columns [jb, jb + N) at plane g (terrain domains)
template <typename R, int N>
__device__ __forceinline__ void ter_factors(const Dev<R>& d, int g, int jb, Arr<R, N>& az, Arr<R, N>& zy) {
    const size_t o = static_cast<size_t>(g) * d.NJP + jb;
    az = ldn<R, N>(d.azT + o);
    zy = ldn<R, N>(d.zyT + o);
}

// -------------------------------------------------- pressure increment parts
// PML part of the air pressure increment of N columns [jb, jb+N) of row i
// (air::cal_fp, air.cpp:1953-2322): per active layer its sigma / beta terms
// with the Q-slab forward differences, then the pairwise corner products,
// added to dp in the reference's order. x and z layers are uniform over the
// columns; the y layer is per column (ysp), all active columns on side ysv
// (1 or 2). Columns outside the y layer take zero y coefficients, which
// adds exact zeros; their slab reads stay inside the padded slab row. The
// reference multiplies every term by dt last; here dt (and gamma P0 or the
// averaging factor) is folded into the layer coefficients first, which
// changes only the last bits of the rounding. TER: every Y derivative of a
// slab also takes its z_over_Y part (the slab's Qv at k + 1).
template <typename R, int N, bool TER = false>
__device__ __forceinline__ void pml_dp_v(const Dev<R>& d, int i, int jb, int k, int xs, int ysp, int ysv, int zs,
                                         R ax, const Arr<R, N>& ay, const Arr<R, N>& az, const Arr<R, N>& zy,
                                         const Arr<R, N>& gu, const Arr<R, N>& gv, const Arr<R, N>& gw,
                                         const Arr<R, N>& pn, const PmlC<R>& X, const PmlC<R>& Z, Arr<R, N>& dp) {
    const R gP0 = d.gP0, dt = d.dt;
    const int NJ = d.NJ;
    const R xS = X.s * dt, xF = X.f * gP0 * dt, zS = Z.s * dt, zF = Z.f * gP0 * dt;
    Arr<R, N> dQux{}, dQvx{}, dQwx{}, QpX{}, dQvy{}, dQwy{}, QpY{}, yS{};
    PmlC<R> Y[N];
    if (xs) {
        const Slab<R>& S = d.sl[xs - 1];
        const int q = S.q(i, jb, k);
        const Arr<R, N> u0 = ldn<R, N>(S.rd[0] + q), u1 = ldn<R, N>(S.rd[0] + q + S.jp);
        const Arr<R, N> v0 = ldn<R, N>(S.rd[1] + q);
        const R vn = (jb + N <= NJ - 1) ? S.rd[1][q + N] : R(0);
        const Arr<R, N> w0 = ldn<R, N>(S.rd[2] + q), w1 = ldn<R, N>(S.rd[2] + q + S.ni * S.jp);
        Arr<R, N> vk{};
        if (TER) vk = ldn<R, N>(S.rd[1] + q + S.ni * S.jp);
        if (ysv | zs) QpX = ldn<R, N>(S.rd[3] + q);
#pragma unroll
        for (int e = 0; e < N; ++e) {
            const R v1 = e + 1 < N ? v0.e[e + 1 < N ? e + 1 : 0] : vn;
            dQux.e[e] = ax * (u1.e[e] - u0.e[e]);
            dQvx.e[e] = ay.e[e] * (v1 - v0.e[e]);
            if (TER) dQvx.e[e] += zy.e[e] * (vk.e[e] - v0.e[e]);
            dQwx.e[e] = az.e[e] * (w1.e[e] - w0.e[e]);
            dp.e[e] += xF * gu.e[e] - xS * (pn.e[e] + gP0 * (dQvx.e[e] + dQwx.e[e]));
        }
    }
    sched_fence();
    if (ysv) {
        const Slab<R>& S = d.sl[ysv + 1];
        const int q = S.q(i, jb, k);
        const Arr<R, N> u0 = ldn<R, N>(S.rd[0] + q), u1 = ldn<R, N>(S.rd[0] + q + S.jp);
        const Arr<R, N> v0 = ldn<R, N>(S.rd[1] + q);
        const R vn = ((ysp >> (2 * (N - 1))) & 3) ? S.rd[1][q + N] : R(0);
        const Arr<R, N> w0 = ldn<R, N>(S.rd[2] + q), w1 = ldn<R, N>(S.rd[2] + q + S.ni * S.jp);
        Arr<R, N> vk{};
        if (TER) vk = ldn<R, N>(S.rd[1] + q + S.ni * S.jp);
        if (xs | zs) QpY = ldn<R, N>(S.rd[3] + q);
#pragma unroll
        for (int e = 0; e < N; ++e) {
            Y[e] = pml_y(d, (ysp >> (2 * e)) & 3, jb + e);
            const R v1 = e + 1 < N ? v0.e[e + 1 < N ? e + 1 : 0] : vn;
            const R dQuy = ax * (u1.e[e] - u0.e[e]);
            dQvy.e[e] = ay.e[e] * (v1 - v0.e[e]);
            if (TER) dQvy.e[e] += zy.e[e] * (vk.e[e] - v0.e[e]);
            dQwy.e[e] = az.e[e] * (w1.e[e] - w0.e[e]);
            yS.e[e] = Y[e].s * dt;
            dp.e[e] += (Y[e].f * gP0 * dt) * gv.e[e] - yS.e[e] * (pn.e[e] + gP0 * (dQuy + dQwy.e[e]));
            if (xs)
                dp.e[e] -= QpX.e[e] * (X.s * yS.e[e]) + gP0 * ((X.g * yS.e[e]) * dQux.e[e] + (Y[e].g * xS) * dQvx.e[e]);
        }
    }
    sched_fence();
    if (zs) {
        const Slab<R>& S = d.sl[zs + 3];
        const int q = S.q(i, jb, k);
        const Arr<R, N> u0 = ldn<R, N>(S.rd[0] + q), u1 = ldn<R, N>(S.rd[0] + q + S.jp);
        const Arr<R, N> v0 = ldn<R, N>(S.rd[1] + q);
        const R vn = (jb + N <= NJ - 1) ? S.rd[1][q + N] : R(0);
        Arr<R, N> vk{};
        if (TER) vk = ldn<R, N>(S.rd[1] + q + S.ni * S.jp);
#pragma unroll
        for (int e = 0; e < N; ++e) {
            const R v1 = e + 1 < N ? v0.e[e + 1 < N ? e + 1 : 0] : vn;
            const R dQuz = ax * (u1.e[e] - u0.e[e]);
            R dQvz = ay.e[e] * (v1 - v0.e[e]);
            if (TER) dQvz += zy.e[e] * (vk.e[e] - v0.e[e]);
            dp.e[e] += zF * gw.e[e] - zS * (pn.e[e] + gP0 * (dQuz + dQvz));
            if (xs) dp.e[e] -= QpX.e[e] * (X.s * zS) + gP0 * ((X.g * zS) * dQux.e[e] + (Z.g * xS) * dQwx.e[e]);
            if (ysv)
                dp.e[e] -=
                    QpY.e[e] * (Y[e].s * zS) + gP0 * ((Y[e].g * zS) * dQvy.e[e] + (Z.g * yS.e[e]) * dQwy.e[e]);
        }
    }
}

// Mean-wind part of the air pressure increment at N columns [jb, jb+N) of
// air k: one-sided upwind advection of p and gamma p div U0
// (air.cpp:1953-2322, wind branch). On a terrain-following grid the z
// advection coefficient takes V z_over_Y and dV/dY its z_over_Y part
// (coef3 and Vav_over_Y of the reference's generic form). The
// coefficients come from the host-built tables (d.wt, which hold the
// terrain terms), one load per table (a 16-byte vector where the N columns
// make one); ax is the row's x factor. The tables are 0 outside the
// interior columns and rows, so face columns take no wind term, as in the
// reference.
template <typename R, int N>
__device__ __forceinline__ void wind_dp(const Dev<R>& d, int k, int jb, R ax, const Arr<R, N>& pn,
                                        const Arr<R, N>& pim, const Arr<R, N>& pjm, const Arr<R, N>& pkm,
                                        Arr<R, N>& dp) {
    const R* t = d.wt + k * d.NJP + jb;
    const int S = d.wtS;
    Arr<R, N> c = ldn<R, N>(t);
#pragma unroll
    for (int e = 0; e < N; ++e) dp.e[e] += -(c.e[e] * ax) * (pn.e[e] - pim.e[e]);
    c = ldn<R, N>(t + S);
#pragma unroll
    for (int e = 0; e < N; ++e) dp.e[e] += -c.e[e] * (pn.e[e] - pjm.e[e]);
    c = ldn<R, N>(t + 2 * S);
#pragma unroll
    for (int e = 0; e < N; ++e) dp.e[e] += -c.e[e] * (pn.e[e] - pkm.e[e]);
    c = ldn<R, N>(t + 3 * S);
#pragma unroll
    for (int e = 0; e < N; ++e) dp.e[e] += -pn.e[e] * c.e[e];
}

// New pressure at N interior columns [jb, jb+N) of row i from their stencil
// values: p_n + increment. Air: air::cal_fp (air.cpp:1953-2322); pore:
// porous::cal_fp (porous.cpp:107-143); accumulation:
// calculation_2D::Cal_pressure (calculation_2D.cpp:581-613).
//   u0 v0 w0 pn  the nodes' u, v, w, p_n
//   ui vj wk     u(i+1), v(j+1), w(g+1)
//   pim pjm pkm  p_n(i-1), p_n(j-1), p_n(g-1) (read with wind only)
//   tc           terrain factors and v(g+1) (read with TER only)
// Columns outside 1..NJ-2 (faces, row padding) get values the caller
// discards; every read for them stays in bounds.
// XF: the rarer features (porous inclusions, vectors with columns of both y
// layers) are compiled in; a kernel built without them is used only for
// domains that have none
// PML: the PML terms are compiled in (a kernel built without them runs only
// tiles that hold no PML node)
template <typename R, bool WIND, int N, bool XF = true, bool PML = true, bool TER = false>
__device__ __forceinline__ Arr<R, N> p_vec(const Dev<R>& d, const PlaneC<R>& pc, const RowC<R>& rc, int i, int jb,
                                           const Arr<R, N>& ay, int ysp, const Arr<R, N>& u0, const Arr<R, N>& v0,
                                           const Arr<R, N>& w0, const Arr<R, N>& pn, const Arr<R, N>& ui,
                                           const Arr<R, N>& vj, const Arr<R, N>& wk, const Arr<R, N>& pim,
                                           const Arr<R, N>& pjm, const Arr<R, N>& pkm,
                                           const TerC<R, N>& tc = TerC<R, N>{}) {
    Arr<R, N> gu, gv, gw, out, az;
#pragma unroll
    for (int e = 0; e < N; ++e) {
        az.e[e] = TER ? tc.az.e[e] : pc.az;
        gu.e[e] = rc.ax * (ui.e[e] - u0.e[e]);
        gv.e[e] = ay.e[e] * (vj.e[e] - v0.e[e]);
        if (TER) gv.e[e] += tc.zy.e[e] * (tc.vk.e[e] - v0.e[e]);
        gw.e[e] = az.e[e] * (wk.e[e] - w0.e[e]);
    }
    if (pc.pore) {
#pragma unroll
        for (int e = 0; e < N; ++e) out.e[e] = pn.e[e] - d.pGama * (gu.e[e] + gv.e[e] + gw.e[e]);
        return out;
    }
    Arr<R, N> dp;
#pragma unroll
    for (int e = 0; e < N; ++e) dp.e[e] = -d.gP0dt * (gu.e[e] + gv.e[e] + gw.e[e]);
    if (WIND) wind_dp<R, N>(d, pc.k, jb, rc.ax, pn, pim, pjm, pkm, dp);
    const int ysv = y_common<N>(ysp);
    if (PML && (rc.xs | ysv | pc.zs)) {
        if (!XF || ysv != 3) {
            pml_dp_v<R, N, TER>(d, i, jb, pc.k, rc.xs, ysp, ysv, pc.zs, rc.ax, ay, az, tc.zy, gu, gv, gw, pn, rc.X,
                                pc.Z, dp);
        } else {  // both y layers within N columns (very narrow grids): column by column
#pragma unroll
            for (int e = 0; e < N; ++e) {
                const int s = (ysp >> (2 * e)) & 3;
                Arr<R, 1> dpe = el(dp, e);
                pml_dp_v<R, 1, TER>(d, i, jb + e, pc.k, rc.xs, s, s, pc.zs, rc.ax, el(ay, e), el(az, e), el(tc.zy, e),
                                    el(gu, e), el(gv, e), el(gw, e), el(pn, e), rc.X, pc.Z, dpe);
                dp.e[e] = dpe.e[0];
            }
        }
    }
#pragma unroll
    for (int e = 0; e < N; ++e) out.e[e] = pn.e[e] + dp.e[e];
    if (XF && rc.inmask) {
#pragma unroll
        for (int e = 0; e < N; ++e) {
            const int mv = mask_at(d, i, jb + e, pc.k);
            if (mv == 1) out.e[e] = pn.e[e] - d.m1_gama * (gu.e[e] + gv.e[e] + gw.e[e]);
            if (mv == 2) out.e[e] = pn.e[e] - d.m2_gama * (gu.e[e] + gv.e[e] + gw.e[e]);
        }
    }
    return out;
}

// -------------------------------------------------- velocity increment parts
// PML part of the air velocity increment of N columns (air::cal_fuvw,
// air.cpp:1476-1949); same column conventions and folding of dt as
// pml_dp_v. p0, pim, pjm,
// pkm: the scheme's pressure at the nodes and at i-1, j-1, g-1. qp_old: the
// slabs' Qp buffers still hold the values from before this step's pressure
// update (single-pass form), so the advanced Qp is formed here as
// Qp + dt * p, the expression of air::Update_PML_Qp. TER: the Y derivative
// of Qp takes its z_over_Y part.
template <typename R, int N, bool TER = false>
__device__ __forceinline__ void pml_dvel_v(const Dev<R>& d, int i, int jb, int k, int xs, int ysp, int ysv, int zs,
                                           R ax, const Arr<R, N>& ay, const Arr<R, N>& az, const Arr<R, N>& zy,
                                           const Arr<R, N>& u0, const Arr<R, N>& v0, const Arr<R, N>& w0,
                                           const Arr<R, N>& gpX, const Arr<R, N>& gpY, const Arr<R, N>& gpZ,
                                           const Arr<R, N>& p0, const Arr<R, N>& pim, const Arr<R, N>& pjm,
                                           const Arr<R, N>& pkm, bool qp_old, const PmlC<R>& X, const PmlC<R>& Z,
                                           Arr<R, N>& du, Arr<R, N>& dv, Arr<R, N>& dw) {
    const R A = d.Aav, dt = d.dt;
    const R xS = X.s * dt, zS = Z.s * dt;
    // backward differences of the slab's Qp advanced to this step
    auto bq = [&](const Slab<R>& S, int q, Arr<R, N>& bx, Arr<R, N>& by, Arr<R, N>& bz) {
        const R* Q = S.rd[3];
        const Arr<R, N> q0 = ldn<R, N>(Q + q), qi = ldn<R, N>(Q + q - S.jp), qk = ldn<R, N>(Q + q - S.ni * S.jp);
        const R qjm = jb > S.ja ? Q[q - 1] : R(0);  // column jb-1
#pragma unroll
        for (int e = 0; e < N; ++e) {
            R a = q0.e[e], b = qi.e[e], c = e > 0 ? q0.e[e > 0 ? e - 1 : 0] : qjm, f = qk.e[e];
            if (qp_old) {
                a = a + dt * p0.e[e];
                b = b + dt * pim.e[e];
                c = c + dt * pjm.e[e];
                f = f + dt * pkm.e[e];
            }
            bx.e[e] = ax * (a - b);
            by.e[e] = ay.e[e] * (a - c);
            if (TER) by.e[e] += zy.e[e] * (a - f);
            bz.e[e] = az.e[e] * (a - f);
        }
    };
    Arr<R, N> bxX{}, byX{}, bzX{}, bxY{}, byY{}, bzY{};
    Arr<R, N> QuX{}, QvX{}, QwX{}, QuY{}, QvY{}, QwY{}, yS{};
    PmlC<R> Y[N];
    if (xs) {
        const Slab<R>& S = d.sl[xs - 1];
        const int q = S.q(i, jb, k);
        bq(S, q, bxX, byX, bzX);
        if (ysv | zs) {
            QuX = ldn<R, N>(S.rd[0] + q);
            QvX = ldn<R, N>(S.rd[1] + q);
            QwX = ldn<R, N>(S.rd[2] + q);
        }
#pragma unroll
        for (int e = 0; e < N; ++e) {
            du.e[e] += (X.f * A * dt) * gpX.e[e] - xS * u0.e[e];
            dv.e[e] -= xS * (v0.e[e] + A * byX.e[e]);
            dw.e[e] -= xS * (w0.e[e] + A * bzX.e[e]);
        }
    }
    sched_fence();
    if (ysv) {
        const Slab<R>& S = d.sl[ysv + 1];
        const int q = S.q(i, jb, k);
        bq(S, q, bxY, byY, bzY);
        if (zs) {
            QuY = ldn<R, N>(S.rd[0] + q);
            QvY = ldn<R, N>(S.rd[1] + q);
            QwY = ldn<R, N>(S.rd[2] + q);
        }
#pragma unroll
        for (int e = 0; e < N; ++e) {
            Y[e] = pml_y(d, (ysp >> (2 * e)) & 3, jb + e);
            yS.e[e] = Y[e].s * dt;
            du.e[e] -= yS.e[e] * (u0.e[e] + A * bxY.e[e]);
            dv.e[e] += (Y[e].f * A * dt) * gpY.e[e] - yS.e[e] * v0.e[e];
            dw.e[e] -= yS.e[e] * (w0.e[e] + A * bzY.e[e]);
            if (xs) {
                const R cXY = X.s * yS.e[e];
                du.e[e] -= QuX.e[e] * cXY + (X.g * yS.e[e] * A) * bxX.e[e];
                dv.e[e] -= QvX.e[e] * cXY + (Y[e].g * xS * A) * byX.e[e];
                dw.e[e] -= QwX.e[e] * cXY;
            }
        }
    }
    sched_fence();
    if (zs) {
        const Slab<R>& S = d.sl[zs + 3];
        const int q = S.q(i, jb, k);
        Arr<R, N> bxZ, byZ, bzZ;
        bq(S, q, bxZ, byZ, bzZ);
#pragma unroll
        for (int e = 0; e < N; ++e) {
            du.e[e] -= zS * (u0.e[e] + A * bxZ.e[e]);
            dv.e[e] -= zS * (v0.e[e] + A * byZ.e[e]);
            dw.e[e] += (Z.f * A * dt) * gpZ.e[e] - zS * w0.e[e];
            if (xs) {
                const R cXZ = X.s * zS;
                du.e[e] -= QuX.e[e] * cXZ + (X.g * zS * A) * bxX.e[e];
                dv.e[e] -= QvX.e[e] * cXZ;
                dw.e[e] -= QwX.e[e] * cXZ + (Z.g * xS * A) * bzX.e[e];
            }
            if (ysv) {
                const R cYZ = Y[e].s * zS;
                du.e[e] -= QuY.e[e] * cYZ;
                dv.e[e] -= QvY.e[e] * cYZ + (Y[e].g * zS * A) * byY.e[e];
                dw.e[e] -= QwY.e[e] * cYZ + (Z.g * yS.e[e] * A) * bzY.e[e];
            }
        }
    }
}

// neighbours of u, v, w for the wind advection terms: f(i+1), f(j+1),
// f(g+1) (the reference's forward differences), or f(i-1), f(j-1), f(g-1)
// when d.upwind
template <typename R, int N>
struct WindNb {
    Arr<R, N> ui, uj, uk, vi, vj, vk, wi, wj, wk;
};

// Mean-wind part of the velocity increment at N columns [jb, jb+N) of
// air k (air::cal_fuvw, air.cpp:1476-1949, wind branch): advection of u,
// v, w by the wind (forward differences as the reference, or backward with
// d.upwind) and the shear terms -(v dU/dY + w dU/dZ) and so on, from the
// host-built tables (d.wt, one load per table); ax is the row's x factor.
template <typename R, int N>
__device__ __forceinline__ void wind_dvel(const Dev<R>& d, int k, int jb, R ax, const Arr<R, N>& u0,
                                          const Arr<R, N>& v0, const Arr<R, N>& w0, const WindNb<R, N>& nb,
                                          Arr<R, N>& du, Arr<R, N>& dv, Arr<R, N>& dw) {
    const R* t = d.wt + k * d.NJP + jb;
    const int S = d.wtS;
    const R sgn = d.upwind ? R(1) : R(-1);  // backward differences: (f - f_back) = -(f_back - f)
    Arr<R, N> c = ldn<R, N>(t);
#pragma unroll
    for (int e = 0; e < N; ++e) {
        const R c1 = sgn * (c.e[e] * ax);
        du.e[e] += c1 * (nb.ui.e[e] - u0.e[e]);
        dv.e[e] += c1 * (nb.vi.e[e] - v0.e[e]);
        dw.e[e] += c1 * (nb.wi.e[e] - w0.e[e]);
    }
    c = ldn<R, N>(t + S);
#pragma unroll
    for (int e = 0; e < N; ++e) {
        const R c2 = sgn * c.e[e];
        du.e[e] += c2 * (nb.uj.e[e] - u0.e[e]);
        dv.e[e] += c2 * (nb.vj.e[e] - v0.e[e]);
        dw.e[e] += c2 * (nb.wj.e[e] - w0.e[e]);
    }
    c = ldn<R, N>(t + 2 * S);
#pragma unroll
    for (int e = 0; e < N; ++e) {
        const R c3 = sgn * c.e[e];
        du.e[e] += c3 * (nb.uk.e[e] - u0.e[e]);
        dv.e[e] += c3 * (nb.vk.e[e] - v0.e[e]);
        dw.e[e] += c3 * (nb.wk.e[e] - w0.e[e]);
    }
    Arr<R, N> a = ldn<R, N>(t + 4 * S), b = ldn<R, N>(t + 5 * S);
#pragma unroll
    for (int e = 0; e < N; ++e) du.e[e] += -(v0.e[e] * a.e[e] + w0.e[e] * b.e[e]);
    a = ldn<R, N>(t + 6 * S);
    b = ldn<R, N>(t + 7 * S);
#pragma unroll
    for (int e = 0; e < N; ++e) dv.e[e] += -(v0.e[e] * a.e[e] + w0.e[e] * b.e[e]);
    a = ldn<R, N>(t + 8 * S);
    b = ldn<R, N>(t + 9 * S);
#pragma unroll
    for (int e = 0; e < N; ++e) dw.e[e] += -(v0.e[e] * a.e[e] + w0.e[e] * b.e[e]);
}

template <typename R, int N>
struct Vel {
    Arr<R, N> u, v, w;
};

// New velocity at N interior columns: u_n + increment, with p the pressure
// the scheme prescribes (p_nn for FB_p_v). Air: air::cal_fuvw
// (air.cpp:1476-1949); pore: porous::cal_fuvw (porous.cpp:58-104);
// accumulation: calculation_2D::Cal_velocity (calculation_2D.cpp:548-579).
// Column conventions as p_vec; tc: terrain factors (TER only; its vk is
// unused here).
template <typename R, bool WIND, int N, bool XF = true, bool PML = true, bool TER = false>
__device__ __forceinline__ Vel<R, N> vel_vec(const Dev<R>& d, const PlaneC<R>& pc, const RowC<R>& rc, int i, int jb,
                                             const Arr<R, N>& ay, int ysp, const Arr<R, N>& u0, const Arr<R, N>& v0,
                                             const Arr<R, N>& w0, const Arr<R, N>& p0, const Arr<R, N>& pim,
                                             const Arr<R, N>& pjm, const Arr<R, N>& pkm, const WindNb<R, N>& nb,
                                             bool qp_old, const TerC<R, N>& tc = TerC<R, N>{}) {
    const R ax = rc.ax;
    Arr<R, N> bpi, bpj, bpk, az;
#pragma unroll
    for (int e = 0; e < N; ++e) {
        az.e[e] = TER ? tc.az.e[e] : pc.az;
        bpi.e[e] = p0.e[e] - pim.e[e];
        bpj.e[e] = p0.e[e] - pjm.e[e];
        bpk.e[e] = p0.e[e] - pkm.e[e];
    }
    Arr<R, N> gpX, gpY, gpZ, du, dv, dw;
#pragma unroll
    for (int e = 0; e < N; ++e) {
        gpX.e[e] = ax * bpi.e[e];
        gpY.e[e] = ay.e[e] * bpj.e[e];
        if (TER) gpY.e[e] += tc.zy.e[e] * bpk.e[e];
        gpZ.e[e] = az.e[e] * bpk.e[e];
    }
    Vel<R, N> r;
    if (pc.pore) {
#pragma unroll
        for (int e = 0; e < N; ++e) {
            r.u.e[e] = u0.e[e] + (-d.pIBdtEff * gpX.e[e] + u0.e[e] * d.pInvB - u0.e[e]);
            r.v.e[e] = v0.e[e] + (-d.pIBdtEff * gpY.e[e] + v0.e[e] * d.pInvB - v0.e[e]);
            r.w.e[e] = w0.e[e] + (-d.pIBdtEff * gpZ.e[e] + w0.e[e] * d.pInvB - w0.e[e]);
        }
        return r;
    }
#pragma unroll
    for (int e = 0; e < N; ++e) {
        du.e[e] = -d.Aavdt * gpX.e[e];
        dv.e[e] = -d.Aavdt * gpY.e[e];
        dw.e[e] = -d.Aavdt * gpZ.e[e];
    }
    if (WIND) wind_dvel<R, N>(d, pc.k, jb, ax, u0, v0, w0, nb, du, dv, dw);
    const int ysv = y_common<N>(ysp);
    if (PML && (rc.xs | ysv | pc.zs)) {
        if (!XF || ysv != 3) {
            pml_dvel_v<R, N, TER>(d, i, jb, pc.k, rc.xs, ysp, ysv, pc.zs, ax, ay, az, tc.zy, u0, v0, w0, gpX, gpY,
                                  gpZ, p0, pim, pjm, pkm, qp_old, rc.X, pc.Z, du, dv, dw);
        } else {  // both y layers within N columns (very narrow grids): column by column
#pragma unroll
            for (int e = 0; e < N; ++e) {
                const int s = (ysp >> (2 * e)) & 3;
                Arr<R, 1> due = el(du, e), dve = el(dv, e), dwe = el(dw, e);
                pml_dvel_v<R, 1, TER>(d, i, jb + e, pc.k, rc.xs, s, s, pc.zs, ax, el(ay, e), el(az, e), el(tc.zy, e),
                                      el(u0, e), el(v0, e), el(w0, e), el(gpX, e), el(gpY, e), el(gpZ, e), el(p0, e),
                                      el(pim, e), el(pjm, e), el(pkm, e), qp_old, rc.X, pc.Z, due, dve, dwe);
                du.e[e] = due.e[0];
                dv.e[e] = dve.e[0];
                dw.e[e] = dwe.e[0];
            }
        }
    }
#pragma unroll
    for (int e = 0; e < N; ++e) {
        r.u.e[e] = u0.e[e] + du.e[e];
        r.v.e[e] = v0.e[e] + dv.e[e];
        r.w.e[e] = w0.e[e] + dw.e[e];
    }
    if (XF && rc.inmask) {
#pragma unroll
        for (int e = 0; e < N; ++e) {
            const int mv = mask_at(d, i, jb + e, pc.k);
            if (mv == 1 || mv == 2) {
                const R a = mv == 1 ? d.m1_ibdteff : d.m2_ibdteff, b = mv == 1 ? d.m1_ib : d.m2_ib;
                r.u.e[e] = u0.e[e] + (-a * gpX.e[e] + u0.e[e] * b - u0.e[e]);
                r.v.e[e] = v0.e[e] + (-a * gpY.e[e] + v0.e[e] * b - v0.e[e]);
                r.w.e[e] = w0.e[e] + (-a * gpZ.e[e] + w0.e[e] * b - w0.e[e]);
            }
        }
    }
    return r;
}

// -------------------------------------------------- node-wise front ends
// Pressure at an interior node with every operand read from global memory
// (two-pass form; the terrain factors when the domain has them).
template <typename R, bool WIND>
__device__ R fresh_p(const Dev<R>& d, int i, int j, int g, bool y1_on) {
    using A = Arr<R, 1>;
    const PlaneC<R> pc = plane_c(d, g);
    const RowC<R> rc = row_c(d, pc, i);
    const A ay{{ldg((pc.pore ? d.ayP : d.ayA) + j)}};
    const int ysp = pc.pore ? 0 : y_side(d, j, y1_on);
    const size_t c = d.ix(g, i, j);
    const size_t si = d.NJP, sg = static_cast<size_t>(d.NI) * d.NJP;
    const R* P = d.pold;
    A pim{{R(0)}}, pjm{{R(0)}}, pkm{{R(0)}};
    if (WIND && !pc.pore) {
        pim.e[0] = P[c - si];
        pjm.e[0] = P[c - 1];
        pkm.e[0] = P[c - sg];
    }
    TerC<R, 1> tc{};
    if (d.azT) {
        ter_factors<R, 1>(d, g, j, tc.az, tc.zy);
        tc.vk.e[0] = d.v_in[c + sg];
        return p_vec<R, WIND, 1, true, true, true>(d, pc, rc, i, j, ay, ysp, A{{d.u_in[c]}}, A{{d.v_in[c]}},
                                                   A{{d.w_in[c]}}, A{{P[c]}}, A{{d.u_in[c + si]}}, A{{d.v_in[c + 1]}},
                                                   A{{d.w_in[c + sg]}}, pim, pjm, pkm, tc)
            .e[0];
    }
    return p_vec<R, WIND, 1>(d, pc, rc, i, j, ay, ysp, A{{d.u_in[c]}}, A{{d.v_in[c]}}, A{{d.w_in[c]}}, A{{P[c]}},
                             A{{d.u_in[c + si]}}, A{{d.v_in[c + 1]}}, A{{d.w_in[c + sg]}}, pim, pjm, pkm)
        .e[0];
}

// Velocity at an interior node with the scheme's pressure read from global
// memory and the Qp slabs already advanced (two-pass form).
template <typename R, bool WIND>
__device__ Vel<R, 1> fresh_vel(const Dev<R>& d, int i, int j, int g, bool y1_on) {
    using A = Arr<R, 1>;
    const PlaneC<R> pc = plane_c(d, g);
    const RowC<R> rc = row_c(d, pc, i);
    const A ay{{ldg((pc.pore ? d.ayP : d.ayA) + j)}};
    const int ysp = pc.pore ? 0 : y_side(d, j, y1_on);
    const size_t c = d.ix(g, i, j);
    const size_t si = d.NJP, sg = static_cast<size_t>(d.NI) * d.NJP;
    const R* p = d.p_in;
    WindNb<R, 1> nb{};
    if (WIND && !pc.pore) {
        const size_t ci = d.upwind ? c - si : c + si, cj = d.upwind ? c - 1 : c + 1, ck = d.upwind ? c - sg : c + sg;
        nb = {A{{d.u_in[ci]}}, A{{d.u_in[cj]}}, A{{d.u_in[ck]}}, A{{d.v_in[ci]}}, A{{d.v_in[cj]}},
              A{{d.v_in[ck]}}, A{{d.w_in[ci]}}, A{{d.w_in[cj]}}, A{{d.w_in[ck]}}};
    }
    if (d.azT) {
        TerC<R, 1> tc{};
        ter_factors<R, 1>(d, g, j, tc.az, tc.zy);
        return vel_vec<R, WIND, 1, true, true, true>(d, pc, rc, i, j, ay, ysp, A{{d.u_in[c]}}, A{{d.v_in[c]}},
                                                     A{{d.w_in[c]}}, A{{p[c]}}, A{{p[c - si]}}, A{{p[c - 1]}},
                                                     A{{p[c - sg]}}, nb, false, tc);
    }
    return vel_vec<R, WIND, 1>(d, pc, rc, i, j, ay, ysp, A{{d.u_in[c]}}, A{{d.v_in[c]}}, A{{d.w_in[c]}}, A{{p[c]}},
                               A{{p[c - si]}}, A{{p[c - 1]}}, A{{p[c - sg]}}, nb, false);
}

// ------------------------------------------------ boundary resolution
// Final pressure at any node. Faces copy from the inward neighbour and the
// east face extrapolates 15/8, -5/4, 3/8 (calculation_2D.cpp:646-721), so
// the final value is that of the clamped node (east: the extrapolation of
// the three clamped nodes behind it). Pore nodes clamp only at their own
// south face; the pore's top row is the air's k=1 row.
template <typename R, bool WIND>
__device__ R final_p(const Dev<R>& d, int i, int j, int g, bool y1_on) {
    const int ic = i < 1 ? 1 : (i > d.NI - 2 ? d.NI - 2 : i);
    int gc = g;
    if (g < d.gAir0) {
        if (g == 0) gc = 1;
    } else {
        if (g == d.NG - 1) gc = g - 1;
        else if (d.rigid_south && g == 0) gc = 1;
    }
    const int jc = j < 1 ? 1 : j;
    if (jc == d.NJ - 1) {
        const R a = fresh_p<R, WIND>(d, ic, d.NJ - 2, gc, y1_on);
        const R b = fresh_p<R, WIND>(d, ic, d.NJ - 3, gc, y1_on);
        const R e = fresh_p<R, WIND>(d, ic, d.NJ - 4, gc, y1_on);
        return R(15.0 / 8.0) * a - R(5.0 / 4.0) * b + R(3.0 / 8.0) * e;
    }
    return fresh_p<R, WIND>(d, ic, jc, gc, y1_on);
}

// TDBC normal velocity at east-face node (i, air k), Cal_TDBC
// (calculation_2D.cpp:1019-1028), with the pressure the scheme prescribes.
template <typename R>
__device__ double tdbc_v(const Dev<R>& d, int i, int k, double p) {
    const double* ps = d.psi_in + (static_cast<size_t>(i) * d.Kair + k) * 6;
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 6; ++q) s += d.td_e[q] * ps[q];
    return d.td_den * (p / d.td_z - s);
}

// Update_Psi at east-face node (i, air k) with the node's own TDBC value
// (calculation_2D.cpp:1012-1017)
template <typename R>
__device__ __forceinline__ void psi_update(const Dev<R>& d, int i, int k, double p) {
    const double vt = tdbc_v(d, i, k, p);
    const size_t o = (static_cast<size_t>(i) * d.Kair + k) * 6;
#pragma unroll
    for (int q = 0; q < 6; ++q) d.psi_out[o + q] = d.td_e[q] * d.psi_in[o + q] + d.td_adt[q] * vt;
}

// ------------------------------------------------------------ kernels
// Pressure pass. Also samples receivers (before the step, get_pressure at
// calculation_2D.cpp:387-403) and advances the Qp slabs (air::Update_PML_Qp,
// air.cpp:2388-2439).
template <typename R, bool WIND>
// pass_code: bit 0 = first pass of the step, bit 1 = parity of the step.
// Step counters: the first pass reads counters[par] and publishes the step to
// the second pass through counters[par ^ 1]; the second pass sets
// counters[par] too. A launch never writes a word its own blocks read, and
// after every step counters[next parity] holds the next step index (the
// fused kernel keeps the same invariant).
__global__ void __launch_bounds__(256) k_pressure(__grid_constant__ const Dev<R> d, int pass_code) {
    const int first_pass = pass_code & 1, par = (pass_code >> 1) & 1;
    const int step = first_pass ? d.counters[par] : d.counters[par ^ 1] - 1;
    const bool y1_on = step + 1 >= d.pml_y_time;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    const int g = blockIdx.z;
    if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0) {
        const int t = threadIdx.y * blockDim.x + threadIdx.x;
        if (t < d.nrec && step < d.rec_steps) {
            const long long n = d.rec_node[t];
            double val = 0.0;
            if (n >= 0) val = static_cast<double>(d.pold[n]);
            if (fabs(val) < 1.0e-100) val = 0.0;
            d.rec_out[static_cast<size_t>(step) * d.nrec + t] = val;
        }
        if (t == 0) {
            if (first_pass) d.counters[par ^ 1] = step + 1;
            else d.counters[par] = step + 1;
        }
    }
    if (j >= d.NJ || i >= d.NI) return;
    const R p = final_p<R, WIND>(d, i, j, g, y1_on);
    const size_t c = d.ix(g, i, j);
    d.p_out[c] = p;
    if (!isfinite(static_cast<float>(p))) atomicOr(d.status, 1);
    if (g >= d.gOff) {
        const int k = g - d.gOff;
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            const Slab<R>& S = d.sl[s];
            if (S.ni == 0 || (s == 2 && !y1_on)) continue;
            if (!S.holds_i(i) || !S.holds_j(j) || !S.holds_k(k)) continue;
            const int q = S.q(i, j, k);
            S.wr[3][q] = S.rd[3][q] + d.dt * p;
        }
    }
}

// Velocity pass. Resolves the face sequence per component (air: N, E, W,
// F, B, S; pore: S, E, W, F, B -- airpore.cpp:324-364 and
// calculation_2D.cpp:777-864), the east TDBC (calculation_2D.cpp:986-1017)
// and advances Qu/Qv/Qw (air::Update_PML_Qvw, air.cpp:2323-2386).
template <typename R, bool WIND>
__global__ void __launch_bounds__(256) k_velocity(__grid_constant__ const Dev<R> d, int pass_code) {
    const int first_pass = pass_code & 1, par = (pass_code >> 1) & 1;
    const int step = first_pass ? d.counters[par] : d.counters[par ^ 1] - 1;
    const bool y1_on = step + 1 >= d.pml_y_time;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    const int g = blockIdx.z;
    if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
        if (first_pass) d.counters[par ^ 1] = step + 1;
        else d.counters[par] = step + 1;
    }
    if (j >= d.NJ || i >= d.NI) return;
    const bool pore = g < d.gAir0;
    const bool onF = i == 0, onB = i == d.NI - 1, onW = j == 0, onE = j == d.NJ - 1;
    const bool onS = pore ? (g == 0) : (d.rigid_south && g == 0);
    const bool onN = !pore && g == d.NG - 1;
    // kind per component: 0 fresh at the clamped node, 1 zero, 2 TDBC
    int ku = 0, kv = 0, kw = 0;
    int ii = i, jj = j, gg = g;
    int ti = i, tg = g;  // TDBC evaluation node (east face)
    // walk faces in reverse application order; a component normal to the
    // face becomes 0 (v on east: TDBC), otherwise the node moves inward
    auto face_i = [&](bool on, int inward) {
        if (!on) return;
        if (ku == 0) ku = 1;
        ii = inward;
    };
    auto face_j_west = [&]() {
        if (kv == 0) kv = 1;
        jj = 1;
    };
    auto face_j_east = [&]() {
        if (kv == 0) {
            if (d.tdbc && !pore) { kv = 2; ti = ii; tg = gg; }
            else kv = 1;
        }
        jj = d.NJ - 2;
    };
    auto face_k = [&](bool on, int inward) {
        if (!on) return;
        if (kw == 0) kw = 1;
        gg = inward;
    };
    if (pore) {
        face_i(onB, d.NI - 2);
        face_i(onF, 1);
        if (onW) face_j_west();
        if (onE) face_j_east();
        face_k(onS, 1);
    } else {
        face_k(onS, 1);
        face_i(onB, d.NI - 2);
        face_i(onF, 1);
        if (onW) face_j_west();
        if (onE) face_j_east();
        face_k(onN, d.NG - 2);
    }
    Vel<R, 1> f{};
    if (ku == 0 || kv == 0 || kw == 0) f = fresh_vel<R, WIND>(d, ii, jj, gg, y1_on);
    R u = ku == 0 ? f.u.e[0] : R(0);
    R v = kv == 0 ? f.v.e[0] : R(0);
    R w = kw == 0 ? f.w.e[0] : R(0);
    // The TDBC reads the "nn" pressure (calculation_2D.cpp:1000). With
    // FB_v_p the velocity half step comes first, so on the very first step
    // that buffer has never been written: zero in a zero-initialised start
    // (every later step it equals p_n).
    const bool p_unset = d.fbvp && step == 0;
    if (kv == 2) {
        const double pe = p_unset ? 0.0 : static_cast<double>(d.p_in[d.ix(tg, ti, d.NJ - 1)]);
        v = static_cast<R>(tdbc_v(d, ti, tg - d.gOff, pe));
    }
    const size_t c = d.ix(g, i, j);
    d.u_out[c] = u;
    d.v_out[c] = v;
    d.w_out[c] = w;
    if (g >= d.gOff) {
        const int k = g - d.gOff;
        if (d.tdbc && onE) {  // Update_Psi with this node's own TDBC value
            const double pe = p_unset ? 0.0 : static_cast<double>(d.p_in[c]);
            const double vt = tdbc_v(d, i, k, pe);
            const size_t o = (static_cast<size_t>(i) * d.Kair + k) * 6;
#pragma unroll
            for (int q = 0; q < 6; ++q) d.psi_out[o + q] = d.td_e[q] * d.psi_in[o + q] + d.td_adt[q] * vt;
        }
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            const Slab<R>& S = d.sl[s];
            if (S.ni == 0 || (s == 2 && !y1_on)) continue;
            if (!S.holds_i(i) || !S.holds_j(j) || !S.holds_k(k)) continue;
            const int q = S.q(i, j, k);
            S.wr[0][q] = S.rd[0][q] + d.dt * u;
            S.wr[1][q] = S.rd[1][q] + d.dt * v;
            S.wr[2][q] = S.rd[2][q] + d.dt * w;
        }
    }
}

}  // namespace fdtd

namespace fdtd {

// Moving-frame shift of one j-row in place (calculation_2D::SetMovingFrame,
// calculation_2D.cpp:458-481; air::SetQMove, air.cpp:2522-2729): ascending j
// reads only values ahead of the write position, so one thread per row is
// exact. west_copy repeats p's "p[0] = p[1]" after the shift.
template <typename R>
__global__ void k_shift_rows(R* a, int rows, int nj, int sh, int lead, int tempJ, int J, int west_copy) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    R* row = a + static_cast<size_t>(r) * nj;
    for (int j = 0; j < nj; ++j) {
        if (j < tempJ + 1 && j + lead - 1 < J - 1) row[j] = row[j + sh];
        else if (j >= tempJ + 1) row[j] = R(0);
    }
    if (west_copy) row[0] = row[1];
}

// Impedance ground (extension; the reference's TDBC acts on the east face
// only, calculation_2D.cpp:986-1017). On the rigid south face w(k = 1) is
// the face velocity: the pressure update at k = 1 takes w(2) - w(1) and the
// rigid face holds it by the copy p(0) = p(1). After a step of the FB_p_v
// scheme this kernel sets w(k = 1) at every interior node from the step's
// new pressure p(k = 1) with the east face's recursion and the ground's
// poles: v_n = den (p / Z - sum e_q psi_q) is the velocity into the ground,
// w = -v_n, psi_q <- e_q psi_q + adt_q v_n. The interior node's thread also
// writes the face nodes whose copies (calculation_2D.cpp:777-864, order N E
// W F B S) end up holding its value, and recomputes the PML integral of w
// at every node it writes from the value read this step (air::Update_PML_Qvw,
// air.cpp:2323-2386), so the state equals an in-step override exactly.
struct GroundC {
    double* psi;  // [q][i][j], row pitch NJP, FP64
    double e[6], adt[6], den, Z;
};

template <typename R>
__global__ void __launch_bounds__(256) k_ground_tdbc(__grid_constant__ const Dev<R> d, GroundC gc, int par) {
    const int j = 1 + static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    const int i = 1 + static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y);
    if (j > d.NJ - 2 || i > d.NI - 2) return;
    // after a step counters[next parity] holds the next step index
    const int step = d.counters[par ^ 1] - 1;
    const bool y1_on = step + 1 >= d.pml_y_time;
    const int g = d.gOff + 1;  // air k = 1
    const double p = static_cast<double>(d.p_out[d.ix(g, i, j)]);
    const size_t qs = static_cast<size_t>(d.NI) * d.NJP;
    double* ps = gc.psi + static_cast<size_t>(i) * d.NJP + j;
    double pv[6];
    double mem = 0.0;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        pv[q] = ps[q * qs];
        mem += gc.e[q] * pv[q];
    }
    const double vn = gc.den * (p / gc.Z - mem);
#pragma unroll
    for (int q = 0; q < 6; ++q) ps[q * qs] = gc.e[q] * pv[q] + gc.adt[q] * vn;
    const R wv = static_cast<R>(-vn);
    const int ia = i == 1 ? 0 : i, ib = i == d.NI - 2 ? d.NI - 1 : i;
    const int ja = j == 1 ? 0 : j, jb = j == d.NJ - 2 ? d.NJ - 1 : j;
    for (int ii = ia; ii <= ib; ++ii)
        for (int jj = ja; jj <= jb; ++jj) {
            d.w_out[d.ix(g, ii, jj)] = wv;
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                const Slab<R>& S = d.sl[s];
                if (S.ni == 0 || (s == 2 && !y1_on)) continue;
                if (!S.holds_i(ii) || !S.holds_j(jj) || !S.holds_k(1)) continue;
                const int q = S.q(ii, jj, 1);
                S.wr[2][q] = S.rd[2][q] + d.dt * wv;
            }
        }
}

}  // namespace fdtd
