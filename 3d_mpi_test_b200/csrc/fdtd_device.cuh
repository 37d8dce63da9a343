// Device-side data model and kernels of the B200 FDTD time-marching path.
//
// One device-resident domain. Air and the porous ground layer are stacked
// in ONE column along k ("unified g axis"): the reference keeps them as two
// grids joined by a two-plane overlap copy (calculation_2D.cpp:865-985:
// air k=0 := pore K-2, pore K-1 := air k=1), which is exactly a shared
// node, so each overlap node is stored once.
//
// Layout: SoA, index ((g * NI) + i) * NJ + j, j (range / propagation axis,
// the reference's Y) contiguous.
//
// A forward-backward step (FB_p_v, airpore.cpp:589-614) is two passes:
//   pressure pass  p_nn for every node, Qp slabs, receiver sampling
//   velocity pass  u,v,w_nn for every node, Qu/Qv/Qw slabs, TDBC state
// Boundary nodes are not swept afterwards as in the reference
// (UpdateBC_*, calculation_2D.cpp:646-864); their final value is resolved
// in closed form: the BC sequence only ever copies from the inward
// neighbour, zeroes a normal component, extrapolates (east p) or applies the
// TDBC (east v), so the last face in sequence decides and the chain ends at
// an interior node whose fresh value the owning thread recomputes.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fdtd {

constexpr int kMaxRec = 64;

template <typename R>
struct Slab {
    // storage range of one PML integral slab, in air node indices (k = air k)
    int i0, j0, k0, ni, nj, nk;
    const R* rd[4];  // u v w p  (values read this pass)
    R* wr[4];        // u v w p  (values written this pass; only one kind per pass)
    __device__ __forceinline__ size_t at(int i, int j, int k) const {
        return (static_cast<size_t>(k - k0) * ni + (i - i0)) * nj + (j - j0);
    }
};

template <typename R>
struct Dev {
    int NI, NJ, NG;
    int NJP;     // row pitch of the field arrays (>= NJ; 16-byte rows for bulk copies)
    int porous;  // porous ground stacked below the air
    int gAir0;   // first g owned by the air medium
    int gOff;    // air k = g - gOff
    int Kair;
    int rigid_south;  // air has its own south face (rigid / absorbing)
    int tdbc;         // east face is the 6-pole TDBC
    int fbvp;         // scheme FB_v_p (velocity first)

    // state: "in" = read, "out" = written
    const R *u_in, *v_in, *w_in, *p_in;  // old u,v,w (or new, FB_v_p pressure pass) and the p used
    const R* pold;                       // p_n (pressure pass)
    R *u_out, *v_out, *w_out, *p_out;

    // derivative factors x_over_X*rdx etc. (reference metric x scale)
    const R *axA, *ayA, *axP, *ayP, *azG;

    // air constants
    R dt, gP0dt, gdt, Aavdt, Aav, gP0;
    // pore constants (porous.cpp:40-51)
    R pGama, pInvB, pIBdtEff;

    // PML 1D profiles: sigma, (1 - 1/beta), (1/beta - 1); side 0 none, 1 low, 2 high
    const R *sxI, *fxI, *gxI, *syJ, *fyJ, *gyJ, *szK, *fzK, *gzK;
    const int8_t *sdI, *sdJ, *sdK;
    int pml_y_time;  // y1 PML switches on once the step count reaches this
    Slab<R> sl[6];   // x1 x2 y1 y2 z1 z2 (ni == 0: absent)

    // mean wind, 2D (j, air k): the reference profiles do not depend on X
    const R *Uw, *Vw, *Ww;

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
    int* counters;              // [0] step index seen by pass 1, [1] by pass 2
    int* status;                // bit 0: non-finite pressure seen

    __device__ __forceinline__ size_t ix(int g, int i, int j) const {
        return (static_cast<size_t>(g) * NI + i) * NJP + j;
    }
};

// Reads of the step's input fields (u, v, w and the old pressure) at
// (i, j, g) straight from global memory.
template <typename R>
struct GlobalFields {
    const Dev<R>& d;
    __device__ __forceinline__ R u(int i, int j, int g) const { return d.u_in[d.ix(g, i, j)]; }
    __device__ __forceinline__ R v(int i, int j, int g) const { return d.v_in[d.ix(g, i, j)]; }
    __device__ __forceinline__ R w(int i, int j, int g) const { return d.w_in[d.ix(g, i, j)]; }
    __device__ __forceinline__ R p(int i, int j, int g) const { return d.pold[d.ix(g, i, j)]; }
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

// -------------------------------------------------- fresh interior values
// Pressure at an interior node of either medium: p_n + increment.
// Air: air::cal_fp (air.cpp:1953-2322); pore: porous::cal_fp (porous.cpp:107-143);
// accumulation: calculation_2D::Cal_pressure (calculation_2D.cpp:581-613).
template <typename R, bool WIND, typename F>
__device__ R fresh_p(const Dev<R>& d, const F& f, int i, int j, int g, bool y1_on) {
    const R u0 = f.u(i, j, g), v0 = f.v(i, j, g), w0 = f.w(i, j, g);
    const R az = ldg(d.azG + g);
    const R pn = f.p(i, j, g);
    if (g < d.gAir0) {  // porous ground
        const R ax = ldg(d.axP + i), ay = ldg(d.ayP + j);
        const R div = ax * (f.u(i + 1, j, g) - u0) + ay * (f.v(i, j + 1, g) - v0) + az * (f.w(i, j, g + 1) - w0);
        return pn - d.pGama * div;
    }
    const R ax = ldg(d.axA + i), ay = ldg(d.ayA + j);
    const R gu = ax * (f.u(i + 1, j, g) - u0), gv = ay * (f.v(i, j + 1, g) - v0), gw = az * (f.w(i, j, g + 1) - w0);
    const int k = g - d.gOff;
    const int8_t* m = d.mask;
    if (m && i >= d.mi0 && i <= d.mi1 && j >= d.mj0 && j <= d.mj1 && k >= d.mk0 && k <= d.mk1) {
        const int mv = m[(static_cast<size_t>(k - d.mk0) * (d.mi1 - d.mi0 + 1) + (i - d.mi0)) * (d.mj1 - d.mj0 + 1) +
                         (j - d.mj0)];
        if (mv == 1) return pn - d.m1_gama * (gu + gv + gw);
        if (mv == 2) return pn - d.m2_gama * (gu + gv + gw);
    }
    R dp = -d.gP0dt * (gu + gv + gw);
    if (WIND) {
        const size_t wk = static_cast<size_t>(k) * d.NJ + j, wS = d.NJ;
        const R U = ldg(d.Uw + wk), V = ldg(d.Vw + wk), W = ldg(d.Ww + wk);
        const R pim = f.p(i - 1, j, g), pjm = f.p(i, j - 1, g), pkm = f.p(i, j, g - 1);
        dp += -(U * ax * d.dt) * (pn - pim) - (V * ay * d.dt) * (pn - pjm) - (W * az * d.dt) * (pn - pkm);
        const R dVdY = ay * (ldg(d.Vw + wk + 1) - ldg(d.Vw + wk - 1)) * R(0.5);
        const R dWdZ = az * (ldg(d.Ww + wk + wS) - ldg(d.Ww + wk - wS)) * R(0.5);
        dp += -d.gdt * pn * (dVdY + dWdZ);
    }
    const int xs = d.sdI[i], ys = y_side(d, j, y1_on), zs = d.sdK[k];
    if (xs | ys | zs) {
        const R sx = xs ? ldg(d.sxI + i) : R(0), sy = ys ? ldg(d.syJ + j) : R(0), sz = zs ? ldg(d.szK + k) : R(0);
        const Slab<R>* SX = xs ? &d.sl[xs - 1] : nullptr;
        const Slab<R>* SY = ys ? &d.sl[ys + 1] : nullptr;
        const Slab<R>* SZ = zs ? &d.sl[zs + 3] : nullptr;
        const R gP0 = d.gP0, dt = d.dt;
        size_t qx = 0, qy = 0, qz = 0;
        R dQux = 0, dQvx = 0, dQwx = 0, dQuy = 0, dQvy = 0, dQwy = 0, dQuz = 0, dQvz = 0;
        if (SX) {
            qx = SX->at(i, j, k);
            const int sj = 1, sk = SX->ni * SX->nj, si = SX->nj;
            dQux = ax * (SX->rd[0][qx + si] - SX->rd[0][qx]);
            dQvx = ay * (SX->rd[1][qx + sj] - SX->rd[1][qx]);
            dQwx = az * (SX->rd[2][qx + sk] - SX->rd[2][qx]);
            dp += ldg(d.fxI + i) * gP0 * gu * dt - sx * (pn + gP0 * (dQvx + dQwx)) * dt;
        }
        if (SY) {
            qy = SY->at(i, j, k);
            const int sj = 1, sk = SY->ni * SY->nj, si = SY->nj;
            dQuy = ax * (SY->rd[0][qy + si] - SY->rd[0][qy]);
            dQvy = ay * (SY->rd[1][qy + sj] - SY->rd[1][qy]);
            dQwy = az * (SY->rd[2][qy + sk] - SY->rd[2][qy]);
            dp += ldg(d.fyJ + j) * gP0 * gv * dt - sy * (pn + gP0 * (dQuy + dQwy)) * dt;
            if (SX) {
                dp += -(SX->rd[3][qx] * sx * sy + gP0 * (ldg(d.gxI + i) * sy * dQux + ldg(d.gyJ + j) * sx * dQvx)) * dt;
            }
        }
        if (SZ) {
            qz = SZ->at(i, j, k);
            const int sk = SZ->ni * SZ->nj, si = SZ->nj;
            dQuz = ax * (SZ->rd[0][qz + si] - SZ->rd[0][qz]);
            dQvz = ay * (SZ->rd[1][qz + 1] - SZ->rd[1][qz]);
            (void)sk;
            dp += ldg(d.fzK + k) * gP0 * gw * dt - sz * (pn + gP0 * (dQuz + dQvz)) * dt;
            if (SX) {
                dp += -(SX->rd[3][qx] * sx * sz + gP0 * (ldg(d.gxI + i) * sz * dQux + ldg(d.gzK + k) * sx * dQwx)) * dt;
            }
            if (SY) {
                dp += -(SY->rd[3][qy] * sy * sz + gP0 * (ldg(d.gyJ + j) * sz * dQvy + ldg(d.gzK + k) * sy * dQwy)) * dt;
            }
        }
    }
    return pn + dp;
}

template <typename R>
struct Vel3 {
    R u, v, w;
};

// Velocity at an interior node: u_n + increment, with p = the pressure the
// scheme prescribes (p_nn for FB_p_v). Air: air::cal_fuvw (air.cpp:1476-1949);
// pore: porous::cal_fuvw (porous.cpp:58-104); accumulation:
// calculation_2D::Cal_velocity (calculation_2D.cpp:548-579).
//
// p0, pim, pjm, pkm: the scheme's pressure at the node and its i-1, j-1,
// g-1 neighbours. qp_old: the slabs' Qp buffers still hold the values from
// before this step's pressure update (fused pass), so the advanced Qp is
// formed here as Qp + dt * p, the expression of air::Update_PML_Qp.
template <typename R, bool WIND, typename F>
__device__ Vel3<R> fresh_vel_core(const Dev<R>& d, const F& f, int i, int j, int g, bool y1_on, R p0, R pim, R pjm,
                                  R pkm, bool qp_old) {
    const R u0 = f.u(i, j, g), v0 = f.v(i, j, g), w0 = f.w(i, j, g);
    const R bpi = p0 - pim, bpj = p0 - pjm, bpk = p0 - pkm;
    const R az = ldg(d.azG + g);
    Vel3<R> r;
    if (g < d.gAir0) {
        const R ax = ldg(d.axP + i), ay = ldg(d.ayP + j);
        r.u = u0 + (-d.pIBdtEff * (ax * bpi) + u0 * d.pInvB - u0);
        r.v = v0 + (-d.pIBdtEff * (ay * bpj) + v0 * d.pInvB - v0);
        r.w = w0 + (-d.pIBdtEff * (az * bpk) + w0 * d.pInvB - w0);
        return r;
    }
    const R ax = ldg(d.axA + i), ay = ldg(d.ayA + j);
    const R gpX = ax * bpi, gpY = ay * bpj, gpZ = az * bpk;
    const int k = g - d.gOff;
    const int8_t* m = d.mask;
    if (m && i >= d.mi0 && i <= d.mi1 && j >= d.mj0 && j <= d.mj1 && k >= d.mk0 && k <= d.mk1) {
        const int mv = m[(static_cast<size_t>(k - d.mk0) * (d.mi1 - d.mi0 + 1) + (i - d.mi0)) * (d.mj1 - d.mj0 + 1) +
                         (j - d.mj0)];
        if (mv == 1 || mv == 2) {
            const R a = mv == 1 ? d.m1_ibdteff : d.m2_ibdteff, b = mv == 1 ? d.m1_ib : d.m2_ib;
            r.u = u0 + (-a * gpX + u0 * b - u0);
            r.v = v0 + (-a * gpY + v0 * b - v0);
            r.w = w0 + (-a * gpZ + w0 * b - w0);
            return r;
        }
    }
    R du = -d.Aavdt * gpX, dv = -d.Aavdt * gpY, dw = -d.Aavdt * gpZ;
    if (WIND) {
        const size_t wk = static_cast<size_t>(k) * d.NJ + j, wS = d.NJ;
        const R U = ldg(d.Uw + wk), V = ldg(d.Vw + wk), W = ldg(d.Ww + wk);
        const R c1 = U * ax * d.dt, c2 = V * ay * d.dt, c3 = W * az * d.dt;
        du += -c1 * (f.u(i + 1, j, g) - u0) - c2 * (f.u(i, j + 1, g) - u0) - c3 * (f.u(i, j, g + 1) - u0);
        dv += -c1 * (f.v(i + 1, j, g) - v0) - c2 * (f.v(i, j + 1, g) - v0) - c3 * (f.v(i, j, g + 1) - v0);
        dw += -c1 * (f.w(i + 1, j, g) - w0) - c2 * (f.w(i, j + 1, g) - w0) - c3 * (f.w(i, j, g + 1) - w0);
        const R h = R(0.5);
        const R dUdY = ay * (ldg(d.Uw + wk + 1) - ldg(d.Uw + wk - 1)) * h;
        const R dUdZ = az * (ldg(d.Uw + wk + wS) - ldg(d.Uw + wk - wS)) * h;
        const R dVdY = ay * (ldg(d.Vw + wk + 1) - ldg(d.Vw + wk - 1)) * h;
        const R dVdZ = az * (ldg(d.Vw + wk + wS) - ldg(d.Vw + wk - wS)) * h;
        const R dWdY = ay * (ldg(d.Ww + wk + 1) - ldg(d.Ww + wk - 1)) * h;
        const R dWdZ = az * (ldg(d.Ww + wk + wS) - ldg(d.Ww + wk - wS)) * h;
        du += -(v0 * dUdY + w0 * dUdZ) * d.dt;
        dv += -(v0 * dVdY + w0 * dVdZ) * d.dt;
        dw += -(v0 * dWdY + w0 * dWdZ) * d.dt;
    }
    const int xs = d.sdI[i], ys = y_side(d, j, y1_on), zs = d.sdK[k];
    if (xs | ys | zs) {
        const R sx = xs ? ldg(d.sxI + i) : R(0), sy = ys ? ldg(d.syJ + j) : R(0), sz = zs ? ldg(d.szK + k) : R(0);
        const Slab<R>* SX = xs ? &d.sl[xs - 1] : nullptr;
        const Slab<R>* SY = ys ? &d.sl[ys + 1] : nullptr;
        const Slab<R>* SZ = zs ? &d.sl[zs + 3] : nullptr;
        const R A = d.Aav, dt = d.dt;
        // backward differences of the slab's Qp advanced to this step
        auto bq = [&](const Slab<R>* S, size_t q, R& bx, R& by, R& bz) {
            const R* Q = S->rd[3];
            const size_t sk = static_cast<size_t>(S->ni) * S->nj;
            R q0 = Q[q], qi = Q[q - S->nj], qj = Q[q - 1], qk = Q[q - sk];
            if (qp_old) {
                q0 = q0 + dt * p0;
                qi = qi + dt * pim;
                qj = qj + dt * pjm;
                qk = qk + dt * pkm;
            }
            bx = ax * (q0 - qi);
            by = ay * (q0 - qj);
            bz = az * (q0 - qk);
        };
        R bxX = 0, byX = 0, bzX = 0, bxY = 0, byY = 0, bzY = 0, bxZ = 0, byZ = 0, bzZ = 0;
        size_t qx = 0, qy = 0;
        if (SX) {
            qx = SX->at(i, j, k);
            bq(SX, qx, bxX, byX, bzX);
            du += -sx * u0 * dt + ldg(d.fxI + i) * (A * gpX) * dt;
            dv += -sx * (v0 + A * byX) * dt;
            dw += -sx * (w0 + A * bzX) * dt;
        }
        if (SY) {
            qy = SY->at(i, j, k);
            bq(SY, qy, bxY, byY, bzY);
            du += -sy * (u0 + A * bxY) * dt;
            dv += ldg(d.fyJ + j) * A * gpY * dt - sy * v0 * dt;
            dw += -sy * (w0 + A * bzY) * dt;
            if (SX) {
                du += -(SX->rd[0][qx] * sx * sy + ldg(d.gxI + i) * sy * A * bxX) * dt;
                dv += -(SX->rd[1][qx] * sx * sy + ldg(d.gyJ + j) * sx * A * byX) * dt;
                dw += -SX->rd[2][qx] * sx * sy * dt;
            }
        }
        if (SZ) {
            const size_t qz = SZ->at(i, j, k);
            R bxZ_, byZ_, bzZ_;
            bq(SZ, qz, bxZ_, byZ_, bzZ_);
            bxZ = bxZ_; byZ = byZ_; bzZ = bzZ_;
            du += -sz * (u0 + A * bxZ) * dt;
            dv += -sz * (v0 + A * byZ) * dt;
            dw += ldg(d.fzK + k) * A * gpZ * dt - sz * w0 * dt;
            if (SX) {
                du += -(SX->rd[0][qx] * sx * sz + ldg(d.gxI + i) * sz * A * bxX) * dt;
                dv += -SX->rd[1][qx] * sx * sz * dt;
                dw += -(SX->rd[2][qx] * sx * sz + ldg(d.gzK + k) * sx * A * bzX) * dt;
            }
            if (SY) {
                du += -SY->rd[0][qy] * sy * sz * dt;
                dv += -(SY->rd[1][qy] * sy * sz + ldg(d.gyJ + j) * sz * A * byY) * dt;
                dw += -(SY->rd[2][qy] * sy * sz + ldg(d.gzK + k) * sy * A * bzY) * dt;
            }
        }
    }
    r.u = u0 + du;
    r.v = v0 + dv;
    r.w = w0 + dw;
    return r;
}

// Velocity with the scheme's pressure read from global memory and the Qp
// slabs already advanced (two-pass path).
template <typename R, bool WIND>
__device__ Vel3<R> fresh_vel(const Dev<R>& d, int i, int j, int g, bool y1_on) {
    const R* p = d.p_in;
    return fresh_vel_core<R, WIND>(d, GlobalFields<R>{d}, i, j, g, y1_on, p[d.ix(g, i, j)], p[d.ix(g, i - 1, j)],
                                   p[d.ix(g, i, j - 1)], p[d.ix(g - 1, i, j)], false);
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
        const GlobalFields<R> gf{d};
        const R a = fresh_p<R, WIND>(d, gf, ic, d.NJ - 2, gc, y1_on);
        const R b = fresh_p<R, WIND>(d, gf, ic, d.NJ - 3, gc, y1_on);
        const R e = fresh_p<R, WIND>(d, gf, ic, d.NJ - 4, gc, y1_on);
        return R(15.0 / 8.0) * a - R(5.0 / 4.0) * b + R(3.0 / 8.0) * e;
    }
    return fresh_p<R, WIND>(d, GlobalFields<R>{d}, ic, jc, gc, y1_on);
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
        if (t < d.nrec) {
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
            if (i < S.i0 || i >= S.i0 + S.ni || j < S.j0 || j >= S.j0 + S.nj || k < S.k0 || k >= S.k0 + S.nk) continue;
            const size_t q = S.at(i, j, k);
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
    Vel3<R> f{R(0), R(0), R(0)};
    if (ku == 0 || kv == 0 || kw == 0) f = fresh_vel<R, WIND>(d, ii, jj, gg, y1_on);
    R u = ku == 0 ? f.u : R(0);
    R v = kv == 0 ? f.v : R(0);
    R w = kw == 0 ? f.w : R(0);
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
            if (i < S.i0 || i >= S.i0 + S.ni || j < S.j0 || j >= S.j0 + S.nj || k < S.k0 || k >= S.k0 + S.nk) continue;
            const size_t q = S.at(i, j, k);
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

}  // namespace fdtd
