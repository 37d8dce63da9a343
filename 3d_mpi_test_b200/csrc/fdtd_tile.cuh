// Tiled single-pass forward-backward step (FB_p_v): each thread block owns
// an (i, j, g) tile -- rows [i0, i1), column vectors [v0, v1) and a chunk of
// core planes [c0, c1) -- and marches it plane by plane in g.
//
// Per plane the block's threads compute the new pressure of the tile plus
// one halo row (i0 - 1) and one halo column vector (v0 - 1) into a shared-
// memory slot, pass ONE block barrier, and then the new velocity of the
// tile's own nodes: the node's u, v, w and new pressure stay in registers
// between the two halves, the i-1 and j-1 pressures come from the slot and
// the g-1 pressure is the thread's own from the previous plane. So u, v, w,
// p are read once and written once per cell (the algorithmic minimum), with
// one barrier per plane.
//
// Stencil inputs arrive by TMA: per plane, one 3D tensor copy per field of
// the box rows [i0-1-W, i1+1) x vectors [v0-1-W, v1+1) (W = 1 with wind)
// into a ring of `ns` stages, completing on one mbarrier per stage, issued
// by thread 0 as soon as the block barrier frees a stage. Boxes that reach
// past the domain read zeros (TMA out-of-bounds fill); those values only
// feed nodes whose results the face rules replace. Every wait is bounded.
// Only this GPU's own memory is ever a source; no multicast.
//
// The host cuts the domain into tiles aligned with the PML and PML-storage
// boundaries, so every tile is either LEAN (no PML node, no PML-storage
// node, no face row or column, no inclusion: interior air or porous
// planes) or FULL. FULL = true compiles in the PML terms, slab updates,
// east TDBC, face rows/columns and receivers; the LEAN instantiation has
// none of them and runs in its own launch. Inside a FULL tile the PML
// branches are uniform across warps whose rows share the layer membership.
//
// Face handling is that of the marching kernel (fdtd_march.cuh): a face
// row's thread computes at its clamped stencil row, the west column copies
// column 1, the east column extrapolates the pressure (15/8, -5/4, 3/8) and
// takes the TDBC or a zero normal velocity, planes 0 and NG-1 are copies of
// planes 1 and NG-2 emitted by their owners.
#pragma once

#include <cuda.h>

#include "fdtd_async.cuh"
#include "fdtd_device.cuh"
#include "fdtd_march.cuh"

namespace fdtd {

constexpr int kTileMaxThreads = 384;

// block timeline (Dev::trace): step slots and tile kinds (0 generic, 1 lean,
// 2 + LM PML / face)
constexpr int kTraceSteps = 64;
constexpr int kTraceKinds = 10;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// thread 0 of a block records its span [t0, now] for tile kind `kind` of the
// step this launch computes
template <typename R>
__device__ __forceinline__ void trace_block(const Dev<R>& d, int par, int kind, unsigned long long t0) {
    if (threadIdx.x != 0 || d.trace == nullptr) return;
    const unsigned long long t1 = global_ns();
    const int step = d.counters[par & 1];
    unsigned long long* s = d.trace + (static_cast<size_t>(step % kTraceSteps) * kTraceKinds + kind) * 4;
    atomicMin(s, t0);
    atomicMax(s + 1, t1);
    atomicAdd(s + 2, t1 - t0);
    atomicAdd(s + 3, 1ull);
}

// output rows, column vectors and core planes of one tile
struct TileBox {
    int i0, i1, v0, v1, c0, c1;
};

// launch-wide tile geometry (every tile of a launch fits it)
struct TileGeo {
    int TI, TV;       // most rows / column vectors of a tile
    int ns;           // ring stages
    int srows, svec;  // staged rows TI + 2 + W, staged column vectors TV + 2 + W
    int box;          // elements of one staged field box (128-byte multiple)
    int pslot;        // elements of one new-pressure slot: (TI + 1) x (TV + 1) vectors
    int ring_off;     // byte offset of the ring in shared memory
};

// tensor maps of u, v, w, p of the time level read this step
struct TileMaps {
    CUtensorMap f[4];
};

// dynamic shared memory of the tiled kernel: TMA destinations are
// 128-byte aligned offsets from this base
__device__ __forceinline__ unsigned char* tile_smem_base() {
    extern __shared__ __align__(1024) unsigned char fdtd_tile_smem[];
    return fdtd_tile_smem;
}

// 3D tiled TMA load (x = column, y = row, z = plane) of this GPU's memory
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// TER: terrain-following grid (per-column z_over_Z and z_over_Y factors)
// Wind advection neighbours of a thread's column vector at plane g from the
// staged boxes: forward (i+1, j+1, g+1; the reference's differences) or,
// with upwind, backward (i-1, j-1, g-1). U, Vf, Wf point at the node in the
// plane-g box, Un.. / Um.. at it in the g+1 / g-1 boxes, SP is the staged
// row pitch; tail: column jb + V exists (forward j neighbour of the last
// element).
template <typename R, int V>
__device__ __forceinline__ WindNb<R, V> wind_nb(bool upwind, const R* U, const R* Vf, const R* Wf, const R* Un,
                                                const R* Vn, const R* Wn, const R* Um, const R* Vm, const R* Wm,
                                                int SP, const Arr<R, V>& u0, const Arr<R, V>& v0,
                                                const Arr<R, V>& w0, bool tail) {
    WindNb<R, V> nb;
    if (!upwind) {
        nb.ui = ldn<R, V>(U + SP);
        nb.vi = ldn<R, V>(Vf + SP);
        nb.wi = ldn<R, V>(Wf + SP);
        nb.uk = ldn<R, V>(Un);
        nb.vk = ldn<R, V>(Vn);
        nb.wk = ldn<R, V>(Wn);
        const R un = tail ? U[V] : R(0), vv = tail ? Vf[V] : R(0), wn = tail ? Wf[V] : R(0);
#pragma unroll
        for (int e = 0; e < V; ++e) {
            const int e1 = e + 1 < V ? e + 1 : 0;
            nb.uj.e[e] = e + 1 < V ? u0.e[e1] : un;
            nb.vj.e[e] = e + 1 < V ? v0.e[e1] : vv;
            nb.wj.e[e] = e + 1 < V ? w0.e[e1] : wn;
        }
    } else {
        nb.ui = ldn<R, V>(U - SP);
        nb.vi = ldn<R, V>(Vf - SP);
        nb.wi = ldn<R, V>(Wf - SP);
        nb.uk = ldn<R, V>(Um);
        nb.vk = ldn<R, V>(Vm);
        nb.wk = ldn<R, V>(Wm);
        const R up = U[-1], vp = Vf[-1], wp = Wf[-1];
#pragma unroll
        for (int e = 0; e < V; ++e) {
            const int e1 = e > 0 ? e - 1 : 0;
            nb.uj.e[e] = e > 0 ? u0.e[e1] : up;
            nb.vj.e[e] = e > 0 ? v0.e[e1] : vp;
            nb.wj.e[e] = e > 0 ? w0.e[e1] : wp;
        }
    }
    return nb;
}

template <typename R, bool WIND, int VW, bool FULL, bool XF, bool TER = false>
__global__ void __launch_bounds__(kTileMaxThreads)
    k_tile(const __grid_constant__ Dev<R> d, const __grid_constant__ TileMaps maps, const TileGeo tg,
           const TileBox* __restrict__ work, int par) {
    static_assert(VW * sizeof(R) == 16, "a thread owns one 16-byte column vector");
    static_assert(FULL || !XF, "the rarer features need the full form");
    constexpr int V = VW;
    constexpr int W = WIND ? 1 : 0;
    const unsigned long long t_start = d.trace ? global_ns() : 0ull;
    const TileBox b = work[blockIdx.x];
    const int NI = d.NI, NJ = d.NJ, NG = d.NG;
    const int TI = tg.TI, TV = tg.TV, ns = tg.ns;
    const int tid = threadIdx.x;
    const int nmain = (TI + 1) * TV;
    const int r = tid < nmain ? tid / TV : tid - nmain;  // 0: halo row i0 - 1
    const int c = tid < nmain ? tid % TV : -1;           // -1: halo column vector v0 - 1
    const int nr = b.i1 - b.i0, nv = b.v1 - b.v0;
    const bool active = tid < nmain + TI + 1 && r <= nr && c < nv && (r > 0 || b.i0 > 0) && (c >= 0 || b.v0 > 0);
    const bool emits = active && r > 0 && c >= 0;
    const int i = b.i0 - 1 + r;
    const int ic = min(max(i, 1), NI - 2);  // stencil row (face rows: the clamped row)
    const int jb = (b.v0 + c) * V;

    // par: bit 0 the step's parity, bit 1 this launch samples the
    // receivers and publishes the step counter (one launch of a step does)
    int step = 0;
    bool y1_on = true;
    if (FULL) {
        step = d.counters[par & 1];
        y1_on = step + 1 >= d.pml_y_time;
        march_bookkeeping(d, par & 1, step, (par & 2) != 0 && blockIdx.x == 0);
    }

    // column data of this thread's vector and row data of its stencil row,
    // fixed for the whole march
    Arr<R, V> ayA{}, ayP{};
    int yside = 0, ystore = 0, ysm1 = 0;
    RowC<R> rcA{}, rcP{};
    bool row_in_mask = false;
    if (active) {
        ayA = ldn<R, V>(d.ayA + jb);
        ayP = ldn<R, V>(d.ayP + jb);
        rcA.ax = ldg(d.axA + ic);
        rcP.ax = ldg(d.axP + ic);
        if (FULL) {
#pragma unroll
            for (int e = 0; e < V; ++e) {
                const int j = jb + e;
                if (j < NJ) {
                    yside |= y_side(d, j, y1_on) << (2 * e);
                    int st = 0;
                    if (d.sl[2].ni && y1_on && d.sl[2].holds_j(j)) st |= 1;
                    if (d.sl[3].ni && d.sl[3].holds_j(j)) st |= 2;
                    ystore |= st << (2 * e);
                }
            }
            ysm1 = jb >= 1 ? y_side(d, jb - 1, y1_on) : 0;
            rcA.xs = d.sdI[ic];
            if (rcA.xs) rcA.X = {ldg(d.sxI + ic), ldg(d.fxI + ic), ldg(d.gxI + ic)};
            row_in_mask = XF && d.mask != nullptr && ic >= d.mi0 && ic <= d.mi1;
        }
    }

    // shared memory: [ns mbarriers | 3 new-pressure slots | ring]
    unsigned char* smem = tile_smem_base();
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    R* pb = reinterpret_cast<R*>(smem + 128);
    R* ring = reinterpret_cast<R*>(smem + tg.ring_off);
    const int SP = tg.svec * V;                                    // staged row pitch
    const int so = (ic - (b.i0 - 1 - W)) * SP + (c + 1 + W) * V;  // this node in a staged box
    const int PR = (TV + 1) * V;                                   // pressure-slot row pitch
    const int po = r * PR + (c + 1) * V;                           // this node in a slot
    const int poi = (ic - b.i0) * PR + (c + 1) * V;                // stencil row - 1 in a slot
    auto fld = [&](int stage, int f) { return ring + static_cast<size_t>(stage * 4 + f) * tg.box; };
    auto pslot = [&](int g) { return pb + (g % 3) * tg.pslot; };

    const int c0 = b.c0, c1 = b.c1;
    const int first = c0 == 1 ? 1 : c0 - 1;  // first plane whose pressure is computed
    const int plo = first - W;                // first staged plane
    const uint32_t stage_bytes = static_cast<uint32_t>(4 * tg.srows * tg.svec * V * sizeof(R));
    if (tid == 0) {
        for (int s = 0; s < ns; ++s) mbar_init(&bar[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    // planes plo, plo + 1, ... are staged in that order into stages 0, 1,
    // ..., ns - 1, 0, ...: stage (x - plo) % ns, its mbarrier in phase
    // ((x - plo) / ns) & 1; the counters below step through both without
    // dividing by the runtime ns
    int ist = 0;  // stage of the next plane issued (thread 0)
    auto issue = [&](int x) {  // plane x into stage ist
        const int s = ist;
        ist = ist + 1 == ns ? 0 : ist + 1;
        fence_proxy_async();
        mbar_arrive_expect_tx(&bar[s], stage_bytes);
        for (int f = 0; f < 4; ++f) tma_load_3d(fld(s, f), &maps.f[f], (b.v0 - 1 - W) * V, b.i0 - 1 - W, x, &bar[s]);
    };
    // A wait that runs out marks the block failed: that thread skips its
    // later waits, and thread 0 issues no more copies, so every stage keeps
    // at most one copy in flight for the drain at the end.
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
    // planes below g are never read after the barrier of plane g, so a stage
    // is refilled once the plane it held is below the plane just passed
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
        if (g == first)
            for (int x = plo; x <= g + 1; ++x) wait_next();
        else
            wait_next();  // plane g + 1
        const int sn = sg + 1 == ns ? 0 : sg + 1, sm = WIND ? (sg == 0 ? ns - 1 : sg - 1) : 0;
        const PlaneC<R> pc = plane_c(d, g);
        const Arr<R, V> ay = pc.pore ? ayP : ayA;
        const int ys = pc.pore ? 0 : yside;
        RowC<R> rc = pc.pore ? rcP : rcA;
        rc.inmask = pc.inmask && row_in_mask;
        Arr<R, V> u0{}, v0{}, w0{}, pnew{}, ui{}, wk{};
        R vn = R(0);
        TerC<R, V> tc{};
        if (TER && active) ter_factors<R, V>(d, g, jb, tc.az, tc.zy);
        // ---- new pressure of the tile and its halos at plane g
        if (active) {
            const R *U = fld(sg, 0) + so, *Vf = fld(sg, 1) + so, *Wf = fld(sg, 2) + so, *P = fld(sg, 3) + so;
            if (TER) tc.vk = ldn<R, V>(fld(sn, 1) + so);
            u0 = ldn<R, V>(U);
            v0 = ldn<R, V>(Vf);
            w0 = ldn<R, V>(Wf);
            const Arr<R, V> pn = ldn<R, V>(P);
            ui = ldn<R, V>(U + SP);
            wk = ldn<R, V>(fld(sn, 2) + so);
            vn = Vf[V];
            Arr<R, V> vj, pim{}, pjm{}, pkm{};
#pragma unroll
            for (int e = 0; e < V; ++e) vj.e[e] = e + 1 < V ? v0.e[e + 1 < V ? e + 1 : 0] : vn;
            if (WIND && !pc.pore) {
                pim = ldn<R, V>(P - SP);
                pkm = ldn<R, V>(fld(sm, 3) + so);
                const R pj0 = P[-1];
#pragma unroll
                for (int e = 0; e < V; ++e) pjm.e[e] = e > 0 ? pn.e[e > 0 ? e - 1 : 0] : pj0;
            }
            pnew = p_vec<R, WIND, V, XF, FULL, TER>(d, pc, rc, ic, jb, ay, ys, u0, v0, w0, pn, ui, vj, wk, pim, pjm,
                                                    pkm, tc);
            if (FULL) {  // west face copies column 1; the east face is extrapolated where it is used
#pragma unroll
                for (int e = 0; e < V; ++e)
                    if (jb + e < 1 || jb + e > NJ - 2) pnew.e[e] = R(0);
                if (jb == 0) pnew.e[0] = pnew.e[1];
            }
            stn<R, V>(pslot(g) + po, pnew);
            if (g == 1) {  // plane 0 (south face) holds plane 1's pressure
                stn<R, V>(pslot(0) + po, pnew);
                pprev = pnew;
            }
        }
        __syncthreads();
        if (tid == 0) refill(g);
        // ---- new velocity and outputs of the tile's own nodes at plane g
        if (emits && g >= c0) {
            const R* Pb = pslot(g);
            const Arr<R, V> Pi = ldn<R, V>(Pb + poi);
            const R Pj0 = jb >= 1 ? Pb[po - 1] : R(0);
            Arr<R, V> Pj;
#pragma unroll
            for (int e = 0; e < V; ++e) Pj.e[e] = e > 0 ? pnew.e[e > 0 ? e - 1 : 0] : Pj0;
            WindNb<R, V> nb{};
            if (WIND && !pc.pore)
                nb = wind_nb<R, V>(d.upwind != 0, fld(sg, 0) + so, fld(sg, 1) + so, fld(sg, 2) + so, fld(sn, 0) + so,
                                   fld(sn, 1) + so, fld(sn, 2) + so, fld(sm, 0) + so, fld(sm, 1) + so,
                                   fld(sm, 2) + so, SP, u0, v0, w0, jb + V <= NJ - 1);
            const Vel<R, V> vel = vel_vec<R, WIND, V, XF, FULL, TER>(d, pc, rc, ic, jb, ay, ys, u0, v0, w0, pnew, Pi,
                                                                      Pj, pprev, nb, true, tc);
            const size_t go = (static_cast<size_t>(g) * NI + i) * d.NJP + jb;
            if (!FULL) {
                stn<R, V>(d.p_out + go, pnew);
                stn<R, V>(d.u_out + go, vel.u);
                stn<R, V>(d.v_out + go, vel.v);
                stn<R, V>(d.w_out + go, vel.w);
#pragma unroll
                for (int e = 0; e < V; ++e) bad += pnew.e[e] * R(0);
                const Arr<R, V> zero{};
                if (g == 1) {  // south face plane: p, u, v of plane 1, w = 0
                    const size_t g0 = static_cast<size_t>(i) * d.NJP + jb;
                    stn<R, V>(d.p_out + g0, pnew);
                    stn<R, V>(d.u_out + g0, vel.u);
                    stn<R, V>(d.v_out + g0, vel.v);
                    stn<R, V>(d.w_out + g0, zero);
                }
                if (g == NG - 2) {  // north face plane
                    const size_t gT = (static_cast<size_t>(NG - 1) * NI + i) * d.NJP + jb;
                    stn<R, V>(d.p_out + gT, pnew);
                    stn<R, V>(d.u_out + gT, vel.u);
                    stn<R, V>(d.v_out + gT, vel.v);
                    stn<R, V>(d.w_out + gT, zero);
                }
            } else {
                Arr<R, V> fu{}, fv{}, fw{};
#pragma unroll
                for (int e = 0; e < V; ++e)
                    if (jb + e >= 1 && jb + e <= NJ - 2) {
                        fu.e[e] = vel.u.e[e];
                        fv.e[e] = vel.v.e[e];
                        fw.e[e] = vel.w.e[e];
                    }
                // west face column: tangential u, w of column 1, normal v = 0
                if (jb == 0) {
                    fu.e[0] = fu.e[1];
                    fw.e[0] = fw.e[1];
                }
                // east face column: tangential u, w of column NJ-2; pressure
                // extrapolated from columns NJ-2..NJ-4 of this row's slot
                // (face rows hold their clamped row's values); v = 0 or TDBC
                const int eE = NJ - 1 - jb;
                const bool hasE = eE >= 0 && eE < V;
                R pE = R(0);
                if (hasE) {
                    if (eE >= 1) {
#pragma unroll
                        for (int e = 1; e < V; ++e)
                            if (e == eE) {
                                fu.e[e] = fu.e[e - 1];
                                fw.e[e] = fw.e[e - 1];
                            }
                    } else if (east_scalar<R, XF>()) {  // column NJ-2 lies in the previous vector
                        using A = Arr<R, 1>;
                        const R *U = fld(sg, 0) + so - 1, *Vf = fld(sg, 1) + so - 1, *Wf = fld(sg, 2) + so - 1;
                        WindNb<R, 1> nbs{};
                        if (WIND && !pc.pore)
                            nbs = wind_nb<R, 1>(d.upwind != 0, U, Vf, Wf, fld(sn, 0) + so - 1, fld(sn, 1) + so - 1,
                                                fld(sn, 2) + so - 1, fld(sm, 0) + so - 1, fld(sm, 1) + so - 1,
                                                fld(sm, 2) + so - 1, SP, A{{U[0]}}, A{{Vf[0]}}, A{{Wf[0]}}, true);
                        const R ays = ldg((pc.pore ? d.ayP : d.ayA) + NJ - 2);
                        TerC<R, 1> tcs{};
                        if (TER) ter_factors<R, 1>(d, g, NJ - 2, tcs.az, tcs.zy);
                        const Vel<R, 1> s = vel_vec<R, WIND, 1, XF, FULL, TER>(
                            d, pc, rc, ic, NJ - 2, A{{ays}}, pc.pore ? 0 : ysm1, A{{U[0]}}, A{{Vf[0]}}, A{{Wf[0]}},
                            A{{Pb[po - 1]}}, A{{Pb[poi - 1]}}, A{{Pb[po - 2]}}, A{{pslot(g - 1)[po - 1]}}, nbs, true,
                            tcs);
                        fu.e[0] = s.u.e[0];
                        fw.e[0] = s.w.e[0];
                    }
                    const R* prow = Pb + r * PR - (b.v0 - 1) * V;  // column j of this row at prow[j]
                    pE = R(15.0 / 8.0) * prow[NJ - 2] - R(5.0 / 4.0) * prow[NJ - 3] + R(3.0 / 8.0) * prow[NJ - 4];
                }
                // front / back faces (rows 0, NI-1): normal u = 0
                if (i == 0 || i == NI - 1) fu = Arr<R, V>{};
                Arr<R, V> pv = pnew;
                if (hasE) {
#pragma unroll
                    for (int e = 0; e < V; ++e)
                        if (e == eE) pv.e[e] = pE;
                }
                const bool tdE = XF && hasE && d.tdbc && !pc.pore;
                if (tdE) {
                    const R vt = static_cast<R>(tdbc_v(d, ic, pc.k, static_cast<double>(pE)));
#pragma unroll
                    for (int e = 0; e < V; ++e)
                        if (e == eE) fv.e[e] = vt;
                }
#pragma unroll
                for (int e = 0; e < V; ++e) bad += pv.e[e] * R(0);
                stn<R, V>(d.p_out + go, pv);
                stn<R, V>(d.u_out + go, fu);
                stn<R, V>(d.v_out + go, fv);
                stn<R, V>(d.w_out + go, fw);
                if (g >= d.gOff) march_slabs<R, V>(d, i, jb, pc.k, ystore, pv, fu, fv, fw);
                if (XF && hasE && d.tdbc && g >= d.gOff) psi_update(d, i, pc.k, static_cast<double>(pE));
                const Arr<R, V> zero{};
                if (g == 1) {  // south face plane: p, u, v of plane 1, w = 0
                    const size_t g0 = static_cast<size_t>(i) * d.NJP + jb;
                    stn<R, V>(d.p_out + g0, pv);
                    stn<R, V>(d.u_out + g0, fu);
                    stn<R, V>(d.v_out + g0, fv);
                    stn<R, V>(d.w_out + g0, zero);
                    if (0 >= d.gOff) {
                        march_slabs<R, V>(d, i, jb, -d.gOff, ystore, pv, fu, fv, zero);
                        if (XF && hasE && d.tdbc) psi_update(d, i, -d.gOff, static_cast<double>(pE));
                    }
                }
                if (g == NG - 2) {  // north face plane: p, u, v of plane NG-2 (east: TDBC on the face row), w = 0
                    const int kT = NG - 1 - d.gOff;
                    const size_t gT = (static_cast<size_t>(NG - 1) * NI + i) * d.NJP + jb;
                    Arr<R, V> vT = fv;
                    if (tdE) {
                        const R vt = static_cast<R>(tdbc_v(d, ic, kT, static_cast<double>(pE)));
#pragma unroll
                        for (int e = 0; e < V; ++e)
                            if (e == eE) vT.e[e] = vt;
                    }
                    stn<R, V>(d.p_out + gT, pv);
                    stn<R, V>(d.u_out + gT, fu);
                    stn<R, V>(d.v_out + gT, vT);
                    stn<R, V>(d.w_out + gT, zero);
                    march_slabs<R, V>(d, i, jb, kT, ystore, pv, fu, vT, zero);
                    if (XF && hasE && d.tdbc) psi_update(d, i, kT, static_cast<double>(pE));
                }
            }
        }
        pprev = pnew;
        sg = sn;
    }
    if (!(bad == R(0))) atomicOr(d.status, 1);
    if (timed_out) atomicOr(d.status, 2);
    // let every copy this block issued land before the block exits (bounded)
    if (tid == 0)
        for (int x = max(plo, issued_hi - ns + 1); x <= issued_hi; ++x)
            mbar_wait(&bar[(x - plo) % ns], static_cast<uint32_t>(((x - plo) / ns) & 1));
    trace_block(d, par, FULL ? 0 : 1, t_start);
}

}  // namespace fdtd
