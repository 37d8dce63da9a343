// Tiled FB_p_v kernel for every tile that holds no inclusion and no TDBC
// node: the PML layers with their edges and corners, the six faces, the
// porous ground and the air/porous interface planes. The generic full-tile
// kernel (fdtd_tile.cuh) keeps domains with inclusions, the east TDBC, or
// an east-face column that starts a column vector (its velocity copies a
// column another thread owns); interior tiles with none of the above run
// the lean form of that kernel.
//
// Marching, staging and thread mapping are those of k_tile. The PML terms
// (air::cal_fp / cal_fuvw, air.cpp:1953-2322 / 1476-1949) of the layers in
// LM (bit 0 x, bit 1 y, bit 2 z) are compiled in, corner products only
// where two layers are; which layer a node is in is decided per thread
// (its row: x, its columns: y) and per plane (z), so layer membership is
// uniform across a warp except at an x-layer edge inside a tile. The layer
// coefficients of the thread's row and columns are fixed for the march.
// Every slab word a plane needs is loaded before the plane's mbarrier wait
// and pressure phase, so the loads overlap the pressure computation and
// the block barrier, and each word is read once per plane (the pressure
// terms, the velocity terms and the slab update share them).
//
// The face rules are those of k_tile: a face row's thread computes at its
// clamped stencil row and zeroes u (front / back), the west column copies
// column 1 (pressure, u, w; v = 0), the east column extrapolates the
// pressure and copies u, w of column NJ-2 (v = 0), planes 0 and NG-1 are
// copies of planes 1 and NG-2 with w = 0, emitted by their owners. Slab updates
// (air::Update_PML_Qp / Qvw, air.cpp:2323-2439) are march_slabs's: Q += dt *
// new value over every slab whose storage holds the output node.
#pragma once

#include "fdtd_tile.cuh"

namespace fdtd {

enum : int { kLmX = 1, kLmY = 2, kLmZ = 4 };

// old slab words of one layer around a node (this step's read buffer)
template <typename R, int V>
struct SlabVals {
    Arr<R, V> u0, u1, v0, w0, w1, p0, pi, pk;  // Qu, Qu(i+1), Qv, Qw, Qw(k+1), Qp, Qp(i-1), Qp(k-1)
    Arr<R, V> vk;                               // Qv(k+1) (terrain: the z_over_Y part of dQv/dY)
    R vn, pj;                                   // Qv(j+V), Qp(j-1)
};

// Loads the words of layer axis AX (0 x, 1 y, 2 z) that a node in the
// layer reads; CORNER: another layer is compiled in (corner products need
// more words); TER: terrain-following grid (every Y derivative of a slab
// also differences it along k); vel: the thread also computes the node's
// velocity; vn_ok: column jb+V may be read.
template <typename R, int V, int AX, bool CORNER, bool TER>
__device__ __forceinline__ void slab_load(const Slab<R>& S, int q, int jb, bool vel, bool vn_ok, SlabVals<R, V>& s) {
    const int si = S.jp, sk = S.ni * S.jp;
    s.u0 = ldn<R, V>(S.rd[0] + q);
    s.v0 = ldn<R, V>(S.rd[1] + q);
    s.w0 = ldn<R, V>(S.rd[2] + q);
    s.p0 = ldn<R, V>(S.rd[3] + q);
    if (AX != 0 || CORNER) s.u1 = ldn<R, V>(S.rd[0] + q + si);
    if (AX != 1 || CORNER) s.vn = vn_ok ? S.rd[1][q + V] : R(0);
    if (AX != 2) s.w1 = ldn<R, V>(S.rd[2] + q + sk);
    if (TER && (AX != 1 || CORNER)) s.vk = ldn<R, V>(S.rd[1] + q + sk);
    if (vel) {
        if (AX != 0 || CORNER) s.pi = ldn<R, V>(S.rd[3] + q - si);
        if (AX != 1 || CORNER) s.pj = jb > S.ja ? S.rd[3][q - 1] : R(0);
        if (AX != 2 || TER) s.pk = ldn<R, V>(S.rd[3] + q - sk);
    }
}

// slab update of one slab at output node offset q over the columns in emask
template <typename R, int V>
__device__ __forceinline__ void slab_store(const Slab<R>& S, int q, int emask, R dt, const Arr<R, V>& ou,
                                           const Arr<R, V>& ov, const Arr<R, V>& ow, const Arr<R, V>& op,
                                           const Arr<R, V>& u, const Arr<R, V>& v, const Arr<R, V>& w,
                                           const Arr<R, V>& p) {
    Arr<R, V> a = ou, b = ov, c = ow, f = op;
#pragma unroll
    for (int e = 0; e < V; ++e)
        if ((emask >> e) & 1) {
            a.e[e] = a.e[e] + dt * u.e[e];
            b.e[e] = b.e[e] + dt * v.e[e];
            c.e[e] = c.e[e] + dt * w.e[e];
            f.e[e] = f.e[e] + dt * p.e[e];
        }
    stn<R, V>(S.wr[0] + q, a);
    stn<R, V>(S.wr[1] + q, b);
    stn<R, V>(S.wr[2] + q, c);
    stn<R, V>(S.wr[3] + q, f);
}

// TER: terrain-following grid (per-column z_over_Z and z_over_Y factors).
// The body of the kernels below: d and maps are the launch's grid
// constants (the bulk copies address the tensor maps in place).
template <typename R, bool WIND, int LM, bool TER>
__device__ __forceinline__ void tile_pml_body(const Dev<R>& d, const TileMaps& maps, const TileGeo& tg,
                                              const TileBox* __restrict__ work, int par) {
    constexpr int V = static_cast<int>(16 / sizeof(R));
    constexpr int W = WIND ? 1 : 0;
    constexpr bool HX = (LM & kLmX) != 0, HY = (LM & kLmY) != 0, HZ = (LM & kLmZ) != 0;
    constexpr bool CX = HX && (HY || HZ), CY = HY && (HX || HZ), CZ = HZ && (HX || HY);  // corner words
    const unsigned long long t_start = d.trace ? global_ns() : 0ull;
    const TileBox b = work[blockIdx.x];
    const int NI = d.NI, NJ = d.NJ, NG = d.NG;
    const int TV = tg.TV, ns = tg.ns;
    const int tid = threadIdx.x;
    const int nmain = (tg.TI + 1) * TV;
    const int r = tid < nmain ? tid / TV : tid - nmain;  // 0: halo row i0 - 1
    const int c = tid < nmain ? tid % TV : -1;           // -1: halo column vector v0 - 1
    const int nr = b.i1 - b.i0, nv = b.v1 - b.v0;
    const bool active =
        tid < nmain + tg.TI + 1 && r <= nr && c < nv && (r > 0 || b.i0 > 0) && (c >= 0 || b.v0 > 0);
    const bool emits = active && r > 0 && c >= 0;
    const int i = b.i0 - 1 + r;
    const int ic = min(max(i, 1), NI - 2);  // stencil row (face rows: the clamped row)
    const int jb = (b.v0 + c) * V;
    // par: bit 0 the step's parity, bit 1 this launch samples the
    // receivers and publishes the step counter (one launch of a step does)
    const int step = d.counters[par & 1];
    const bool y1_on = step + 1 >= d.pml_y_time;
    march_bookkeeping(d, par & 1, step, (par & 2) != 0 && blockIdx.x == 0);
    const R dt = d.dt, gP0 = d.gP0, A = d.Aav;
    const bool vn_ok = jb + V <= NJ - 1;

    // fixed for the march: factors of the thread's row and columns, and the
    // x / y layer and storage membership with the layer coefficients
    Arr<R, V> ayA{}, ayP{};
    R axA = R(0), axP = R(0);
    int xs = 0, xst = 0;  // x layer side of the stencil row; x slab storing the output row (1, 2; 0 none)
    PmlC<R> X{R(0), R(0), R(0)};
    int ysp = 0, ysv = 0, yst = 0, ysm = 0;  // y sides per column, common side, storing slab, its column mask
    Arr<R, V> yS{}, yF{}, yG{};
    if (active) {
        ayA = ldn<R, V>(d.ayA + jb);
        ayP = ldn<R, V>(d.ayP + jb);
        axA = ldg(d.axA + ic);
        axP = ldg(d.axP + ic);
        if (HX) {
            xs = d.sdI[ic];
            if (xs) X = {ldg(d.sxI + ic), ldg(d.fxI + ic), ldg(d.gxI + ic)};
            if (d.sl[0].ni && d.sl[0].holds_i(i)) xst = 1;
            else if (d.sl[1].ni && d.sl[1].holds_i(i)) xst = 2;
        }
        if (HY) {
#pragma unroll
            for (int e = 0; e < V; ++e) {
                const int j = jb + e;
                if (j < NJ) {
                    const int s = y_side(d, j, y1_on);
                    ysp |= s << (2 * e);
                    if (s) {
                        yS.e[e] = ldg(d.syJ + j) * dt;
                        yF.e[e] = ldg(d.fyJ + j);
                        yG.e[e] = ldg(d.gyJ + j);
                    }
                    if (d.sl[2].ni && y1_on && d.sl[2].holds_j(j)) {
                        yst = 1;
                        ysm |= 1 << e;
                    }
                    if (d.sl[3].ni && d.sl[3].holds_j(j)) {
                        yst = 2;
                        ysm |= 1 << e;
                    }
                }
            }
            ysv = y_common<V>(ysp);  // the host keeps vectors with both y layers out of these tiles
        }
    }
    const int live = NJ - jb >= V ? (1 << V) - 1 : (1 << max(NJ - jb, 0)) - 1;  // columns < NJ

    // shared memory: [ns mbarriers | 3 new-pressure slots | ring]
    unsigned char* smem = tile_smem_base();
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    R* pb = reinterpret_cast<R*>(smem + 128);
    R* ring = reinterpret_cast<R*>(smem + tg.ring_off);
    const int SP = tg.svec * V;
    const int so = (ic - (b.i0 - 1 - W)) * SP + (c + 1 + W) * V;
    const int PR = (TV + 1) * V;
    const int po = r * PR + (c + 1) * V;
    const int poi = (ic - b.i0) * PR + (c + 1) * V;
    auto fld = [&](int stage, int f) { return ring + static_cast<size_t>(stage * 4 + f) * tg.box; };
    auto pslot = [&](int g) { return pb + (g % 3) * tg.pslot; };

    const int c0 = b.c0, c1 = b.c1;
    const int first = c0 == 1 ? 1 : c0 - 1;
    const int plo = first - W;
    const uint32_t stage_bytes = static_cast<uint32_t>(4 * tg.srows * tg.svec * V * sizeof(R));
    if (tid == 0) {
        for (int s = 0; s < ns; ++s) mbar_init(&bar[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    // planes plo, plo + 1, ... go to stages 0, 1, ..., ns - 1, 0, ... in
    // order (stage (x - plo) % ns, phase ((x - plo) / ns) & 1), stepped by
    // counters instead of divisions by the runtime ns
    int ist = 0;  // stage of the next plane issued (thread 0)
    auto issue = [&](int x) {
        const int s = ist;
        ist = ist + 1 == ns ? 0 : ist + 1;
        fence_proxy_async();
        mbar_arrive_expect_tx(&bar[s], stage_bytes);
        for (int f = 0; f < 4; ++f) tma_load_3d(fld(s, f), &maps.f[f], (b.v0 - 1 - W) * V, b.i0 - 1 - W, x, &bar[s]);
    };
    bool timed_out = false;
    const long long spin = d.wait_spin;
    int wst = 0;        // stage of the next plane waited for (planes plo, plo + 1, ... in order)
    uint32_t wph = 0;   // its mbarrier phase parity
    auto wait_next = [&]() {
        if (!timed_out && !mbar_wait(&bar[wst], wph, spin)) timed_out = true;
        if (++wst == ns) {
            wst = 0;
            wph ^= 1u;
        }
    };
    int issued_hi = plo - 1;
    // a stage is refilled once no thread reads its plane any more: planes
    // below g after the barrier of plane g, below g - 1 when upwind wind
    // advection reads plane g - 1 in the velocity phase (the host then
    // keeps at least 4 stages)
    const int lag = (WIND && d.upwind) ? 1 : 0;
    auto refill = [&](int g) {
        while (issued_hi + 1 <= c1 && issued_hi + 1 - ns < g - lag && !timed_out) issue(++issued_hi);
    };
    if (tid == 0) refill(plo);

    R bad = R(0);
    Arr<R, V> pprev{};
    int sg = first - plo;  // stage of plane g
    for (int g = first; g < c1; ++g) {
        const int k = g - d.gOff;
        const PlaneC<R> pc = plane_c(d, g);
        const bool pore = pc.pore;
        const R ax = pore ? axP : axA;
        const Arr<R, V> ay = pore ? ayP : ayA;
        const bool vel = emits && g >= c0;
        // layer membership of this node at this plane (PML terms: air only)
        const int xl = HX && !pore ? xs : 0;
        const int yl = HY && !pore ? ysv : 0;
        const int zl = HZ && !pore ? pc.zs : 0;
        const PmlC<R> Z = pc.Z;
        // per-column factors of this plane: z_over_Z * rdz (and on a
        // terrain-following grid z_over_Y * rdz)
        Arr<R, V> az, zy{};
        if (TER && active) ter_factors<R, V>(d, g, jb, az, zy);
        if (!TER) {
#pragma unroll
            for (int e = 0; e < V; ++e) az.e[e] = pc.az;
        }
        // the slab words of the plane, ahead of the staged fields
        SlabVals<R, V> sx{}, sy{}, sz{};
        if (HX && xl) slab_load<R, V, 0, CX, TER>(d.sl[xl - 1], d.sl[xl - 1].q(ic, jb, k), jb, vel, vn_ok, sx);
        if (HY && yl)  // Qv(j+V) of a y slab only where the vector's last column is in the layer
            slab_load<R, V, 1, CY, TER>(d.sl[yl + 1], d.sl[yl + 1].q(ic, jb, k), jb, vel,
                                   vn_ok && ((ysp >> (2 * (V - 1))) & 3) != 0, sy);
        if (HZ && zl) slab_load<R, V, 2, CZ, TER>(d.sl[zl + 3], d.sl[zl + 3].q(ic, jb, k), jb, vel, vn_ok, sz);
        if (g == first)
            for (int x = plo; x <= g + 1; ++x) wait_next();
        else
            wait_next();  // plane g + 1
        const int sn = sg + 1 == ns ? 0 : sg + 1, sm = WIND ? (sg == 0 ? ns - 1 : sg - 1) : 0;
        Arr<R, V> u0{}, v0{}, w0{}, pnew{}, ui{}, wk{}, gu{}, gv{}, gw{};
        R vn = R(0);
        // ---- new pressure of the tile and its halos at plane g
        if (active) {
            const R *U = fld(sg, 0) + so, *Vf = fld(sg, 1) + so, *Wf = fld(sg, 2) + so, *P = fld(sg, 3) + so;
            u0 = ldn<R, V>(U);
            v0 = ldn<R, V>(Vf);
            w0 = ldn<R, V>(Wf);
            const Arr<R, V> pn = ldn<R, V>(P);
            ui = ldn<R, V>(U + SP);
            wk = ldn<R, V>(fld(sn, 2) + so);
            vn = Vf[V];
            Arr<R, V> vk{};
            if (TER) vk = ldn<R, V>(fld(sn, 1) + so);
#pragma unroll
            for (int e = 0; e < V; ++e) {
                const R vj = e + 1 < V ? v0.e[e + 1 < V ? e + 1 : 0] : vn;
                gu.e[e] = ax * (ui.e[e] - u0.e[e]);
                gv.e[e] = ay.e[e] * (vj - v0.e[e]);
                if (TER) gv.e[e] += zy.e[e] * (vk.e[e] - v0.e[e]);
                gw.e[e] = az.e[e] * (wk.e[e] - w0.e[e]);
            }
            Arr<R, V> dp;
            if (pore) {
#pragma unroll
                for (int e = 0; e < V; ++e) dp.e[e] = -d.pGama * (gu.e[e] + gv.e[e] + gw.e[e]);
            } else {
#pragma unroll
                for (int e = 0; e < V; ++e) dp.e[e] = -d.gP0dt * (gu.e[e] + gv.e[e] + gw.e[e]);
                if (WIND) {
                    const Arr<R, V> pim = ldn<R, V>(P - SP), pkm = ldn<R, V>(fld(sm, 3) + so);
                    const R pj0 = P[-1];
                    Arr<R, V> pjm;
#pragma unroll
                    for (int e = 0; e < V; ++e) pjm.e[e] = e > 0 ? pn.e[e > 0 ? e - 1 : 0] : pj0;
                    wind_dp<R, V>(d, k, jb, ax, pn, pim, pjm, pkm, dp);
                }
                // PML terms in the order of pml_dp_v: x, y (with x-y
                // corners), z (with x-z and y-z corners)
                const R xS = X.s * dt, zS = Z.s * dt;
                Arr<R, V> dQux{}, dQvx{}, dQwx{}, dQvy{}, dQwy{};
                if (HX && xl) {
                    const R xF = X.f * gP0 * dt;
#pragma unroll
                    for (int e = 0; e < V; ++e) {
                        const R v1 = e + 1 < V ? sx.v0.e[e + 1 < V ? e + 1 : 0] : sx.vn;
                        if (CX) dQux.e[e] = ax * (sx.u1.e[e] - sx.u0.e[e]);
                        dQvx.e[e] = ay.e[e] * (v1 - sx.v0.e[e]);
                        if (TER) dQvx.e[e] += zy.e[e] * (sx.vk.e[e] - sx.v0.e[e]);
                        dQwx.e[e] = az.e[e] * (sx.w1.e[e] - sx.w0.e[e]);
                        dp.e[e] += xF * gu.e[e] - xS * (pn.e[e] + gP0 * (dQvx.e[e] + dQwx.e[e]));
                    }
                }
                if (HY && yl) {
#pragma unroll
                    for (int e = 0; e < V; ++e) {
                        const R v1 = e + 1 < V ? sy.v0.e[e + 1 < V ? e + 1 : 0] : sy.vn;
                        const R dQuy = ax * (sy.u1.e[e] - sy.u0.e[e]);
                        if (CY) {
                            dQvy.e[e] = ay.e[e] * (v1 - sy.v0.e[e]);
                            if (TER) dQvy.e[e] += zy.e[e] * (sy.vk.e[e] - sy.v0.e[e]);
                        }
                        dQwy.e[e] = az.e[e] * (sy.w1.e[e] - sy.w0.e[e]);
                        dp.e[e] += (yF.e[e] * gP0 * dt) * gv.e[e] - yS.e[e] * (pn.e[e] + gP0 * (dQuy + dQwy.e[e]));
                        if (HX && xl)
                            dp.e[e] -= sx.p0.e[e] * (X.s * yS.e[e]) +
                                       gP0 * ((X.g * yS.e[e]) * dQux.e[e] + (yG.e[e] * xS) * dQvx.e[e]);
                    }
                }
                if (HZ && zl) {
                    const R zF = Z.f * gP0 * dt;
#pragma unroll
                    for (int e = 0; e < V; ++e) {
                        const R v1 = e + 1 < V ? sz.v0.e[e + 1 < V ? e + 1 : 0] : sz.vn;
                        const R dQuz = ax * (sz.u1.e[e] - sz.u0.e[e]);
                        R dQvz = ay.e[e] * (v1 - sz.v0.e[e]);
                        if (TER) dQvz += zy.e[e] * (sz.vk.e[e] - sz.v0.e[e]);
                        dp.e[e] += zF * gw.e[e] - zS * (pn.e[e] + gP0 * (dQuz + dQvz));
                        if (HX && xl)
                            dp.e[e] -= sx.p0.e[e] * (X.s * zS) +
                                       gP0 * ((X.g * zS) * dQux.e[e] + (Z.g * xS) * dQwx.e[e]);
                        if (HY && yl)
                            dp.e[e] -= sy.p0.e[e] * (yS.e[e] * Z.s) +
                                       gP0 * ((yG.e[e] * zS) * dQvy.e[e] + (Z.g * yS.e[e]) * dQwy.e[e]);
                    }
                }
            }
#pragma unroll
            for (int e = 0; e < V; ++e) pnew.e[e] = jb + e <= NJ - 2 ? pn.e[e] + dp.e[e] : R(0);
            // west face copies column 1; the east face (past NJ-2) is
            // extrapolated where it is emitted
            if (jb == 0) pnew.e[0] = pnew.e[1];
            stn<R, V>(pslot(g) + po, pnew);
            if (g == 1) {  // plane 0 (south face) holds plane 1's pressure
                stn<R, V>(pslot(0) + po, pnew);
                pprev = pnew;
            }
        }
        __syncthreads();
        if (tid == 0) refill(g);
        // ---- new velocity and outputs of the tile's own nodes at plane g
        if (vel) {
            const R* Pb = pslot(g);
            const Arr<R, V> Pi = ldn<R, V>(Pb + poi);
            const R Pj0 = jb >= 1 ? Pb[po - 1] : R(0);
            Arr<R, V> Pj, gpX, gpY, gpZ, du, dv, dw, nu, nv, nw;
#pragma unroll
            for (int e = 0; e < V; ++e) {
                Pj.e[e] = e > 0 ? pnew.e[e > 0 ? e - 1 : 0] : Pj0;
                gpX.e[e] = ax * (pnew.e[e] - Pi.e[e]);
                gpY.e[e] = ay.e[e] * (pnew.e[e] - Pj.e[e]);
                if (TER) gpY.e[e] += zy.e[e] * (pnew.e[e] - pprev.e[e]);
                gpZ.e[e] = az.e[e] * (pnew.e[e] - pprev.e[e]);
            }
            if (pore) {
#pragma unroll
                for (int e = 0; e < V; ++e) {
                    nu.e[e] = u0.e[e] + (-d.pIBdtEff * gpX.e[e] + u0.e[e] * d.pInvB - u0.e[e]);
                    nv.e[e] = v0.e[e] + (-d.pIBdtEff * gpY.e[e] + v0.e[e] * d.pInvB - v0.e[e]);
                    nw.e[e] = w0.e[e] + (-d.pIBdtEff * gpZ.e[e] + w0.e[e] * d.pInvB - w0.e[e]);
                }
            } else {
#pragma unroll
                for (int e = 0; e < V; ++e) {
                    du.e[e] = -d.Aavdt * gpX.e[e];
                    dv.e[e] = -d.Aavdt * gpY.e[e];
                    dw.e[e] = -d.Aavdt * gpZ.e[e];
                }
                if (WIND) {
                    const WindNb<R, V> nb =
                        wind_nb<R, V>(d.upwind != 0, fld(sg, 0) + so, fld(sg, 1) + so, fld(sg, 2) + so,
                                      fld(sn, 0) + so, fld(sn, 1) + so, fld(sn, 2) + so, fld(sm, 0) + so,
                                      fld(sm, 1) + so, fld(sm, 2) + so, SP, u0, v0, w0, jb + V <= NJ - 1);
                    wind_dvel<R, V>(d, k, jb, ax, u0, v0, w0, nb, du, dv, dw);
                }
                // PML terms in the order of pml_dvel_v, with Qp advanced to
                // this step at the node and its backward neighbours
                // (air::Update_PML_Qp folded in: Qp + dt p)
                const R xS = X.s * dt, zS = Z.s * dt;
#pragma unroll
                for (int e = 0; e < V; ++e) {
                    const R dp0 = dt * pnew.e[e], dpi = dt * Pi.e[e], dpj = dt * Pj.e[e], dpk = dt * pprev.e[e];
                    R bxX = R(0), byX = R(0), bzX = R(0);
                    if (HX && xl) {
                        const R a = sx.p0.e[e] + dp0;
                        if (CX) bxX = ax * (a - (sx.pi.e[e] + dpi));
                        const R fk = sx.pk.e[e] + dpk;
                        byX = ay.e[e] * (a - ((e > 0 ? sx.p0.e[e > 0 ? e - 1 : 0] : sx.pj) + dpj));
                        if (TER) byX += zy.e[e] * (a - fk);
                        bzX = az.e[e] * (a - fk);
                        du.e[e] += (X.f * A * dt) * gpX.e[e] - xS * u0.e[e];
                        dv.e[e] -= xS * (v0.e[e] + A * byX);
                        dw.e[e] -= xS * (w0.e[e] + A * bzX);
                    }
                    R byY = R(0), bzY = R(0);
                    if (HY && yl) {
                        const R a = sy.p0.e[e] + dp0;
                        const R bxY = ax * (a - (sy.pi.e[e] + dpi));
                        const R fk = sy.pk.e[e] + dpk;
                        if (CY) {
                            byY = ay.e[e] * (a - ((e > 0 ? sy.p0.e[e > 0 ? e - 1 : 0] : sy.pj) + dpj));
                            if (TER) byY += zy.e[e] * (a - fk);
                        }
                        bzY = az.e[e] * (a - fk);
                        du.e[e] -= yS.e[e] * (u0.e[e] + A * bxY);
                        dv.e[e] += (yF.e[e] * A * dt) * gpY.e[e] - yS.e[e] * v0.e[e];
                        dw.e[e] -= yS.e[e] * (w0.e[e] + A * bzY);
                        if (HX && xl) {
                            const R cXY = X.s * yS.e[e];
                            du.e[e] -= sx.u0.e[e] * cXY + (X.g * yS.e[e] * A) * bxX;
                            dv.e[e] -= sx.v0.e[e] * cXY + (yG.e[e] * xS * A) * byX;
                            dw.e[e] -= sx.w0.e[e] * cXY;
                        }
                    }
                    if (HZ && zl) {
                        const R a = sz.p0.e[e] + dp0;
                        const R bxZ = ax * (a - (sz.pi.e[e] + dpi));
                        R byZ = ay.e[e] * (a - ((e > 0 ? sz.p0.e[e > 0 ? e - 1 : 0] : sz.pj) + dpj));
                        if (TER) byZ += zy.e[e] * (a - (sz.pk.e[e] + dpk));
                        du.e[e] -= zS * (u0.e[e] + A * bxZ);
                        dv.e[e] -= zS * (v0.e[e] + A * byZ);
                        dw.e[e] += (Z.f * A * dt) * gpZ.e[e] - zS * w0.e[e];
                        if (HX && xl) {
                            const R cXZ = X.s * zS;
                            du.e[e] -= sx.u0.e[e] * cXZ + (X.g * zS * A) * bxX;
                            dv.e[e] -= sx.v0.e[e] * cXZ;
                            dw.e[e] -= sx.w0.e[e] * cXZ + (Z.g * xS * A) * bzX;
                        }
                        if (HY && yl) {
                            const R cYZ = yS.e[e] * Z.s;
                            du.e[e] -= sy.u0.e[e] * cYZ;
                            dv.e[e] -= sy.v0.e[e] * cYZ + (yG.e[e] * zS * A) * byY;
                            dw.e[e] -= sy.w0.e[e] * cYZ + (Z.g * yS.e[e] * A) * bzY;
                        }
                    }
                }
#pragma unroll
                for (int e = 0; e < V; ++e) {
                    nu.e[e] = u0.e[e] + du.e[e];
                    nv.e[e] = v0.e[e] + dv.e[e];
                    nw.e[e] = w0.e[e] + dw.e[e];
                }
            }
            // faces: west column (tangential u, w of column 1, v = 0), east
            // column (u, w of column NJ-2, v = 0, pressure extrapolated
            // 15/8, -5/4, 3/8 from columns NJ-2..NJ-4 of this row's slot;
            // the host runs the east TDBC and an east column that starts a
            // vector in the generic kernel), front / back rows (u = 0)
#pragma unroll
            for (int e = 0; e < V; ++e)
                if (jb + e > NJ - 2) {
                    nu.e[e] = R(0);
                    nv.e[e] = R(0);
                    nw.e[e] = R(0);
                }
            if (jb == 0) {
                nu.e[0] = nu.e[1];
                nv.e[0] = R(0);
                nw.e[0] = nw.e[1];
            }
            Arr<R, V> pv = pnew;
            const int eE = NJ - 1 - jb;
            if (eE >= 1 && eE < V) {
                const R* prow = Pb + r * PR - (b.v0 - 1) * V;  // column j of this row at prow[j]
                const R pE = R(15.0 / 8.0) * prow[NJ - 2] - R(5.0 / 4.0) * prow[NJ - 3] + R(3.0 / 8.0) * prow[NJ - 4];
#pragma unroll
                for (int e = 1; e < V; ++e)
                    if (e == eE) {
                        nu.e[e] = nu.e[e - 1];
                        nw.e[e] = nw.e[e - 1];
                        pv.e[e] = pE;
                    }
            }
            if (i == 0 || i == NI - 1) nu = Arr<R, V>{};
#pragma unroll
            for (int e = 0; e < V; ++e) bad += pv.e[e] * R(0);
            const size_t go = (static_cast<size_t>(g) * NI + i) * d.NJP + jb;
            stn<R, V>(d.p_out + go, pv);
            stn<R, V>(d.u_out + go, nu);
            stn<R, V>(d.v_out + go, nv);
            stn<R, V>(d.w_out + go, nw);
            const Arr<R, V> zero{};
            // slab updates of this node and of the face plane it emits
            auto slabs_at = [&](int kk, const Arr<R, V>& p, const Arr<R, V>& u, const Arr<R, V>& v,
                                const Arr<R, V>& w, bool own) {
                // own: the node of this plane, whose old slab words are
                // already loaded when its stencil row is its output row
                if (HX && xst) {
                    const Slab<R>& S = d.sl[xst - 1];
                    const int q = S.q(i, jb, kk);
                    if (own && xl && i == ic) slab_store<R, V>(S, q, live, dt, sx.u0, sx.v0, sx.w0, sx.p0, u, v, w, p);
                    else
                        slab_store<R, V>(S, q, live, dt, ldn<R, V>(S.rd[0] + q), ldn<R, V>(S.rd[1] + q),
                                         ldn<R, V>(S.rd[2] + q), ldn<R, V>(S.rd[3] + q), u, v, w, p);
                }
                if (HY && yst) {
                    const Slab<R>& S = d.sl[yst + 1];
                    const int q = S.q(i, jb, kk);
                    if (own && yl && i == ic) slab_store<R, V>(S, q, ysm, dt, sy.u0, sy.v0, sy.w0, sy.p0, u, v, w, p);
                    else
                        slab_store<R, V>(S, q, ysm, dt, ldn<R, V>(S.rd[0] + q), ldn<R, V>(S.rd[1] + q),
                                         ldn<R, V>(S.rd[2] + q), ldn<R, V>(S.rd[3] + q), u, v, w, p);
                }
                if (HZ) {
                    int zst = 0;
                    if (d.sl[4].ni && d.sl[4].holds_k(kk)) zst = 1;
                    else if (d.sl[5].ni && d.sl[5].holds_k(kk)) zst = 2;
                    if (zst) {
                        const Slab<R>& S = d.sl[zst + 3];
                        const int q = S.q(i, jb, kk);
                        if (own && zl == zst && i == ic)
                            slab_store<R, V>(S, q, live, dt, sz.u0, sz.v0, sz.w0, sz.p0, u, v, w, p);
                        else
                            slab_store<R, V>(S, q, live, dt, ldn<R, V>(S.rd[0] + q), ldn<R, V>(S.rd[1] + q),
                                             ldn<R, V>(S.rd[2] + q), ldn<R, V>(S.rd[3] + q), u, v, w, p);
                    }
                }
            };
            if (g >= d.gOff) slabs_at(k, pv, nu, nv, nw, true);
            if (g == 1) {  // south face plane: p, u, v of plane 1, w = 0
                const size_t g0 = static_cast<size_t>(i) * d.NJP + jb;
                stn<R, V>(d.p_out + g0, pv);
                stn<R, V>(d.u_out + g0, nu);
                stn<R, V>(d.v_out + g0, nv);
                stn<R, V>(d.w_out + g0, zero);
                if (0 >= d.gOff) slabs_at(-d.gOff, pv, nu, nv, zero, false);
            }
            if (g == NG - 2) {  // north face plane: p, u, v of plane NG-2, w = 0
                const size_t gT = (static_cast<size_t>(NG - 1) * NI + i) * d.NJP + jb;
                stn<R, V>(d.p_out + gT, pv);
                stn<R, V>(d.u_out + gT, nu);
                stn<R, V>(d.v_out + gT, nv);
                stn<R, V>(d.w_out + gT, zero);
                slabs_at(NG - 1 - d.gOff, pv, nu, nv, zero, false);
            }
        }
        pprev = pnew;
        sg = sn;
    }
    if (!(bad == R(0))) atomicOr(d.status, 1);
    if (timed_out) atomicOr(d.status, 2);
    if (tid == 0)
        for (int x = max(plo, issued_hi - ns + 1); x <= issued_hi; ++x)
            mbar_wait(&bar[(x - plo) % ns], static_cast<uint32_t>(((x - plo) / ns) & 1));
    trace_block(d, par, 2 + LM, t_start);
}

// Without wind the kernel of a single layer (or none) is capped at 128
// registers: four 128-thread blocks fit an SM instead of three, with no
// spill (+3 % FP32, +2 % FP64 on the porous-hill domain). The kinds of two
// or three layers would spill under the cap and keep what they need, as
// does the wind form.
template <typename R, bool WIND, int LM, bool TER = false>
__global__ void __maxnreg__(((LM & (LM - 1)) == 0) ? 128 : 168)
    k_tile_pml_calm(const __grid_constant__ Dev<R> d, const __grid_constant__ TileMaps maps, const TileGeo tg,
                    const TileBox* __restrict__ work, int par) {
    tile_pml_body<R, false, LM, TER>(d, maps, tg, work, par);
}

template <typename R, bool WIND, int LM, bool TER = false>
__global__ void __launch_bounds__(kTileMaxThreads)
    k_tile_pml_wind(const __grid_constant__ Dev<R> d, const __grid_constant__ TileMaps maps, const TileGeo tg,
                    const TileBox* __restrict__ work, int par) {
    tile_pml_body<R, true, LM, TER>(d, maps, tg, work, par);
}

}  // namespace fdtd
