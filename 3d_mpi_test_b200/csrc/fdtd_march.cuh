// Single-pass forward-backward step (FB_p_v): pressure and velocity of a
// plane in ONE marching pass over the unified g axis.
//
// Block = rows [i0, i1) of the i axis x all NJ columns x a chunk of "core"
// planes [c0, c1) within [1, NG-2]. The block marches g upward. For each
// plane it computes the new pressure of its rows plus one halo row below
// (i0-1) into shared memory (two plane slots: g and g-1), then the new
// velocity of its own rows from that shared-memory pressure (backward
// differences in i, j, g) -- so u, v, w, p are read once from HBM and
// written once, instead of the two passes' p round trip. Plane 0 (south
// face: porous or rigid ground) and plane NG-1 (north face) are copies of
// planes 1 and NG-2 (w = 0; east TDBC evaluated on the face row) and are
// emitted by the blocks owning planes 1 and NG-2. The in-plane face walk is
// the two-pass velocity kernel's (fdtd_device.cuh) in closed form.
//
// Stencil inputs stream into a shared-memory ring by 1D bulk copies
// (cp.async.bulk, mbarrier transaction counts): one copy per field per plane
// (the staged rows of a plane are contiguous in global memory), two planes
// ahead of the plane being computed, issued by one thread. Only this GPU's
// own memory is ever a source.
//
// Thread mapping: a thread owns one 16-byte vector of V columns
// [jb, jb + V) for the whole march (its column coefficients and PML-y
// membership stay in registers) and one of `trows` interleaved row
// sequences; every shared and global field access is one 16-byte vector.
//
// Slab buffers: every read uses the values from before this step (Qp is
// advanced on the fly for the velocity stencil as Qp + dt * p, which is
// air::Update_PML_Qp, air.cpp:2388-2439), every write goes to the other
// buffer.
#pragma once

#include "fdtd_async.cuh"
#include "fdtd_device.cuh"

namespace fdtd {

// Whether a kernel form holds the scalar velocity update of an east column
// that starts a vector. The FP32 lean form leaves it out (122 -> 116
// registers with 2-column vectors, about 4% faster on a porous-ground
// domain); the FP64 lean form
// keeps it, because leaving it out measured about 1.5% slower there.
template <typename R, bool XF>
__host__ __device__ constexpr bool east_scalar() { return XF || sizeof(R) == 8; }

struct MarchTiling {
    int TI;        // nominal rows per block (>= 2)
    int nrb;       // row blocks; the last one also takes the remainder rows
    int GC;        // core planes per block
    int nchunk;    // plane chunks
    int rows_max;  // most rows any block owns (shared-memory sizing)
    int nstage;    // bulk-copy ring depth: W + 2 planes in use, the rest in flight
    int trows;     // thread rows: a block is trows x (NJP / VW) threads
    int VW;        // columns per thread
};

__device__ __forceinline__ unsigned char* march_smem() {
    extern __shared__ __align__(16) unsigned char fdtd_smem[];
    return fdtd_smem;
}

// Shared-memory geometry of one block. Offsets are element offsets from the
// ring base (fields) or the pressure base (P). A ring stage holds, per field,
// only the rows the block reads: u rows [iclo, ichi+1], v and w rows
// [iclo, ichi+W], p rows [iclo-W, ichi] (W = 1 with wind), where
// [iclo, ichi] are the clamped stencil rows of the block.
struct MarchGeo {
    int pitch;     // NJP
    int ss;        // one ring stage (elements)
    int fb[4];     // field f, row i, column j of a stage at fb[f] + i * pitch + j
    int r0[4];     // first staged row of field f
    int nrow[4];   // staged rows of field f
    int rlo;       // first pressure row
    int srows;     // rows per pressure slot
    int ns;        // ring stages
    __device__ __forceinline__ int stage(int x) const { return (x % ns) * ss; }
    __device__ __forceinline__ int prow(int slot, int i) const { return (slot * srows + i - rlo) * pitch; }
};

// receivers (calculation_2D::get_pressure on p_n before the step) and the
// step counter: even steps read counters[0] and publish counters[1], odd
// steps the reverse (no block reads the word this launch writes)
template <typename R>
__device__ __forceinline__ void march_bookkeeping(const Dev<R>& d, int par, int step, bool first_block) {
    if (first_block) {
        const int tt = threadIdx.x;
        for (int r = tt; r < d.nrec && step < d.rec_steps; r += blockDim.x) {  // blocks may be narrower than the receiver list
            const long long n = d.rec_node[r];
            double val = 0.0;
            if (n >= 0) val = static_cast<double>(d.pold[n]);
            if (fabs(val) < 1.0e-100) val = 0.0;
            d.rec_out[static_cast<size_t>(step) * d.nrec + r] = val;
        }
        if (tt == 0) d.counters[par ^ 1] = step + 1;
    }
}

// New pressure of the V columns [jb, jb + V) at stencil row ic of plane q
// (staged at ring offset oq; plane q+1 at on, q-1 at om). Interior columns
// 1..NJ-2 are kept; column 0 repeats column 1 (west face copy,
// calculation_2D.cpp:650-660); columns >= NJ-1 are 0 -- the east face is
// extrapolated where it is used.
template <typename R, bool WIND, int VW, bool XF>
__device__ __forceinline__ Arr<R, VW> march_p(const Dev<R>& d, const PlaneC<R>& pc, const RowC<R>& rc, const R* rg,
                                          const MarchGeo& G, int oq, int on, int om, int ic, int jb,
                                          const Arr<R, VW>& ay, int ysp) {
    constexpr int V = VW;
    const int NJ = d.NJ, pitch = G.pitch;
    const int o = oq + ic * pitch + jb;
    const R *U = rg + G.fb[0], *Vf = rg + G.fb[1], *Wf = rg + G.fb[2], *P = rg + G.fb[3];
    const Arr<R, VW> u0 = ldn<R, VW>(U + o), v0 = ldn<R, VW>(Vf + o), w0 = ldn<R, VW>(Wf + o), pn = ldn<R, VW>(P + o);
    const Arr<R, VW> ui = ldn<R, VW>(U + o + pitch);
    const Arr<R, VW> wk = ldn<R, VW>(Wf + on + ic * pitch + jb);
    const R vn = (jb + V <= NJ - 1) ? Vf[o + V] : R(0);
    Arr<R, VW> vj, pim{}, pjm{}, pkm{};
#pragma unroll
    for (int e = 0; e < V; ++e) vj.e[e] = e + 1 < V ? v0.e[e + 1 < V ? e + 1 : 0] : vn;
    if (WIND && !pc.pore) {
        pim = ldn<R, VW>(P + o - pitch);
        pkm = ldn<R, VW>(P + om + ic * pitch + jb);
        const R pj0 = jb >= 1 ? P[o - 1] : R(0);
#pragma unroll
        for (int e = 0; e < V; ++e) pjm.e[e] = e > 0 ? pn.e[e > 0 ? e - 1 : 0] : pj0;
    }
    Arr<R, VW> out = p_vec<R, WIND, VW, XF>(d, pc, rc, ic, jb, ay, ysp, u0, v0, w0, pn, ui, vj, wk, pim, pjm, pkm);
#pragma unroll
    for (int e = 0; e < V; ++e)
        if (jb + e < 1 || jb + e > NJ - 2) out.e[e] = R(0);
    if (jb == 0) out.e[0] = out.e[1];
    return out;
}

// Fresh velocity at stencil node (ii, j) of plane q, every operand loaded
// as a scalar (the east-face column when it starts a new vector).
template <typename R, bool WIND>
__device__ __forceinline__ Vel<R, 1> march_vel_scalar(const Dev<R>& d, const PlaneC<R>& pc, const RowC<R>& rc,
                                                      const R* rg, const R* pb, const MarchGeo& G, int oq, int on,
                                                      int slot, int ii, int j, R ay, int ys) {
    using A = Arr<R, 1>;
    const int pitch = G.pitch;
    const int o = oq + ii * pitch + j;
    const R *U = rg + G.fb[0], *Vf = rg + G.fb[1], *Wf = rg + G.fb[2];
    const int pr = G.prow(slot, ii) + j, pp = G.prow(slot ^ 1, ii) + j;
    WindNb<R, 1> nb{};
    if (WIND && !pc.pore) {
        const int ok = on + ii * pitch + j;
        nb = {A{{U[o + pitch]}},  A{{U[o + 1]}},  A{{U[ok]}},  A{{Vf[o + pitch]}}, A{{Vf[o + 1]}},
              A{{Vf[ok]}},        A{{Wf[o + pitch]}}, A{{Wf[o + 1]}}, A{{Wf[ok]}}};
    }
    return vel_vec<R, WIND, 1>(d, pc, rc, ii, j, A{{ay}}, ys, A{{U[o]}}, A{{Vf[o]}}, A{{Wf[o]}}, A{{pb[pr]}},
                               A{{pb[pr - pitch]}}, A{{pb[pr - 1]}}, A{{pb[pp]}}, nb, true);
}

// PML slab updates at output row i, columns [jb, jb + V), air k: Q += dt *
// new value over every slab whose storage holds the node
// (air::Update_PML_Qp / Update_PML_Qvw, air.cpp:2323-2439). Each slab row
// vector is read, updated in the columns it stores, and written whole to
// the other buffer (padding columns carry over). ystore: per column 2 bits
// (y1, y2 storage).
template <typename R, int VW>
__device__ __forceinline__ void march_slabs(const Dev<R>& d, int i, int jb, int k, int ystore, const Arr<R, VW>& p,
                                            const Arr<R, VW>& u, const Arr<R, VW>& v, const Arr<R, VW>& w) {
    constexpr int V = VW;
    const R dt = d.dt;
    auto put = [&](const Slab<R>& S, int q, int emask) {
        Arr<R, VW> a = ldn<R, VW>(S.rd[0] + q), b = ldn<R, VW>(S.rd[1] + q), c = ldn<R, VW>(S.rd[2] + q), f = ldn<R, VW>(S.rd[3] + q);
#pragma unroll
        for (int e = 0; e < V; ++e)
            if ((emask >> e) & 1) {
                a.e[e] = a.e[e] + dt * u.e[e];
                b.e[e] = b.e[e] + dt * v.e[e];
                c.e[e] = c.e[e] + dt * w.e[e];
                f.e[e] = f.e[e] + dt * p.e[e];
            }
        stn<R, VW>(S.wr[0] + q, a);
        stn<R, VW>(S.wr[1] + q, b);
        stn<R, VW>(S.wr[2] + q, c);
        stn<R, VW>(S.wr[3] + q, f);
    };
    const int n = d.NJ - jb;
    const int live = n >= V ? (1 << V) - 1 : (1 << (n > 0 ? n : 0)) - 1;  // columns < NJ
#pragma unroll
    for (int s = 0; s < 2; ++s) {  // x slabs hold whole rows
        const Slab<R>& S = d.sl[s];
        if (S.ni && S.holds_i(i)) put(S, S.q(i, jb, k), live);
    }
    int m1 = 0, m2 = 0;  // y slabs: membership per column
#pragma unroll
    for (int e = 0; e < V; ++e) {
        m1 |= ((ystore >> (2 * e)) & 1) << e;
        m2 |= ((ystore >> (2 * e + 1)) & 1) << e;
    }
    if (m1) put(d.sl[2], d.sl[2].q(i, jb, k), m1);
    if (m2) put(d.sl[3], d.sl[3].q(i, jb, k), m2);
#pragma unroll
    for (int s = 4; s < 6; ++s) {  // z slabs hold whole planes
        const Slab<R>& S = d.sl[s];
        if (S.ni && S.holds_k(k)) put(S, S.q(i, jb, k), live);
    }
}

// Emit output row i of plane q: new velocity at the clamped stencil row ii
// from the shared-memory pressure, face resolution, outputs, slabs, TDBC
// state, and the face planes 0 / NG-1 next to it.
template <typename R, bool WIND, int VW, bool XF>
__device__ __forceinline__ void march_emit(const Dev<R>& d, const PlaneC<R>& pc, const R* rg, const R* pb,
                                           const MarchGeo& G, int oq, int on, int slot, int q, int i, int jb,
                                           const Arr<R, VW>& ay, int ysp, int ysm1, int ystore, R& bad) {
    constexpr int V = VW;
    const int NI = d.NI, NJ = d.NJ, NG = d.NG, pitch = G.pitch;
    const int ii = i < 1 ? 1 : (i > NI - 2 ? NI - 2 : i);
    const RowC<R> rc = row_c(d, pc, ii);
    const int o = oq + ii * pitch + jb;
    const int pr = G.prow(slot, ii) + jb;
    const R *U = rg + G.fb[0], *Vf = rg + G.fb[1], *Wf = rg + G.fb[2];
    const Arr<R, VW> u0 = ldn<R, VW>(U + o), v0 = ldn<R, VW>(Vf + o), w0 = ldn<R, VW>(Wf + o);
    const Arr<R, VW> P0 = ldn<R, VW>(pb + pr), Pi = ldn<R, VW>(pb + pr - pitch), Pk = ldn<R, VW>(pb + G.prow(slot ^ 1, ii) + jb);
    const R Pj0 = jb >= 1 ? pb[pr - 1] : R(0);
    Arr<R, VW> Pj;
#pragma unroll
    for (int e = 0; e < V; ++e) Pj.e[e] = e > 0 ? P0.e[e > 0 ? e - 1 : 0] : Pj0;
    WindNb<R, VW> nb{};
    if (WIND && !pc.pore) {
        const int ok = on + ii * pitch + jb;
        nb.ui = ldn<R, VW>(U + o + pitch);
        nb.vi = ldn<R, VW>(Vf + o + pitch);
        nb.wi = ldn<R, VW>(Wf + o + pitch);
        nb.uk = ldn<R, VW>(U + ok);
        nb.vk = ldn<R, VW>(Vf + ok);
        nb.wk = ldn<R, VW>(Wf + ok);
        const bool tail = jb + V <= NJ - 1;
        const R un = tail ? U[o + V] : R(0), vn = tail ? Vf[o + V] : R(0), wn = tail ? Wf[o + V] : R(0);
#pragma unroll
        for (int e = 0; e < V; ++e) {
            const int e1 = e + 1 < V ? e + 1 : 0;
            nb.uj.e[e] = e + 1 < V ? u0.e[e1] : un;
            nb.vj.e[e] = e + 1 < V ? v0.e[e1] : vn;
            nb.wj.e[e] = e + 1 < V ? w0.e[e1] : wn;
        }
    }
    const Vel<R, VW> r = vel_vec<R, WIND, VW, XF>(d, pc, rc, ii, jb, ay, ysp, u0, v0, w0, P0, Pi, Pj, Pk, nb, true);
    Arr<R, VW> fu{}, fv{}, fw{};
#pragma unroll
    for (int e = 0; e < V; ++e)
        if (jb + e >= 1 && jb + e <= NJ - 2) {
            fu.e[e] = r.u.e[e];
            fv.e[e] = r.v.e[e];
            fw.e[e] = r.w.e[e];
        }
    // west face column: tangential u, w of column 1, normal v = 0
    if (jb == 0) {
        fu.e[0] = fu.e[1];
        fw.e[0] = fw.e[1];
    }
    // east face column: tangential u, w of column NJ-2, v = 0 or TDBC below
    const int eE = NJ - 1 - jb;
    const bool hasE = eE >= 0 && eE < V;
    const int prow_i = G.prow(slot, i);
    R pE = R(0), pEs = R(0);  // east-face pressure of row i and of the stencil row ii
    if (hasE) {
        if (eE >= 1) {
#pragma unroll
            for (int e = 1; e < V; ++e)
                if (e == eE) {
                    fu.e[e] = fu.e[e - 1];
                    fw.e[e] = fw.e[e - 1];
                }
        } else if (east_scalar<R, XF>()) {  // the east column starts a vector: (NJ - 1) % VW == 0
            const Vel<R, 1> s = march_vel_scalar<R, WIND>(d, pc, rc, rg, pb, G, oq, on, slot, ii, NJ - 2,
                                                          ldg((pc.pore ? d.ayP : d.ayA) + NJ - 2), pc.pore ? 0 : ysm1);
            fu.e[0] = s.u.e[0];
            fw.e[0] = s.w.e[0];
        }
        auto ext = [&](int row) {  // east extrapolation, calculation_2D.cpp:662-672
            return R(15.0 / 8.0) * pb[row + NJ - 2] - R(5.0 / 4.0) * pb[row + NJ - 3] + R(3.0 / 8.0) * pb[row + NJ - 4];
        };
        pE = ext(prow_i);
        pEs = (ii == i) ? pE : ext(G.prow(slot, ii));
    }
    // front / back faces (rows 0, NI-1): normal u = 0
    if (i == 0 || i == NI - 1) fu = Arr<R, VW>{};
    Arr<R, VW> pv = ldn<R, VW>(pb + prow_i + jb);
    if (hasE) {
#pragma unroll
        for (int e = 0; e < V; ++e)
            if (e == eE) pv.e[e] = pE;
    }
    const bool tdE = XF && hasE && d.tdbc && !pc.pore;
    if (tdE) {
        const R vt = static_cast<R>(tdbc_v(d, ii, pc.k, static_cast<double>(pEs)));
#pragma unroll
        for (int e = 0; e < V; ++e)
            if (e == eE) fv.e[e] = vt;
    }
#pragma unroll
    for (int e = 0; e < V; ++e) bad += pv.e[e] * R(0);
    const size_t go = (static_cast<size_t>(q) * NI + i) * pitch + jb;
    stn<R, VW>(d.p_out + go, pv);
    stn<R, VW>(d.u_out + go, fu);
    stn<R, VW>(d.v_out + go, fv);
    stn<R, VW>(d.w_out + go, fw);
    if (q >= d.gOff) march_slabs<R, VW>(d, i, jb, pc.k, ystore, pv, fu, fv, fw);
    if (XF && hasE && d.tdbc && q >= d.gOff) psi_update(d, i, pc.k, static_cast<double>(pE));
    const Arr<R, VW> zero{};
    if (q == 1) {  // south face plane: p, u, v of plane 1, w = 0
        const size_t g0 = static_cast<size_t>(i) * pitch + jb;
        stn<R, VW>(d.p_out + g0, pv);
        stn<R, VW>(d.u_out + g0, fu);
        stn<R, VW>(d.v_out + g0, fv);
        stn<R, VW>(d.w_out + g0, zero);
        if (0 >= d.gOff) {
            march_slabs<R, VW>(d, i, jb, -d.gOff, ystore, pv, fu, fv, zero);
            if (XF && hasE && d.tdbc) psi_update(d, i, -d.gOff, static_cast<double>(pE));
        }
    }
    if (q == NG - 2) {  // north face plane: p, u, v of plane NG-2 (east: TDBC on the face row), w = 0
        const int kT = NG - 1 - d.gOff;
        const size_t gT = (static_cast<size_t>(NG - 1) * NI + i) * pitch + jb;
        Arr<R, VW> vT = fv;
        if (tdE) {
            const R vt = static_cast<R>(tdbc_v(d, ii, kT, static_cast<double>(pEs)));
#pragma unroll
            for (int e = 0; e < V; ++e)
                if (e == eE) vT.e[e] = vt;
        }
        stn<R, VW>(d.p_out + gT, pv);
        stn<R, VW>(d.u_out + gT, fu);
        stn<R, VW>(d.v_out + gT, vT);
        stn<R, VW>(d.w_out + gT, zero);
        march_slabs<R, VW>(d, i, jb, kT, ystore, pv, fu, vT, zero);
        if (XF && hasE && d.tdbc) psi_update(d, i, kT, static_cast<double>(pE));
    }
}

// One block of the march: row block bx, plane chunk by of domain d. A block
// may have more threads than the tile's trows thread rows (batched launches
// over domains of different widths): the extra threads only take part in
// the block barriers.
template <typename R, bool WIND, int VW, bool XF>
__device__ __forceinline__ void march_block(const Dev<R>& d, const MarchTiling& t, int par, int bx, int by) {
    static_assert(VW >= 2 && VW * sizeof(R) <= 16, "a thread owns 2..16 bytes of columns");
    constexpr int V = VW;
    const int NI = d.NI, NJ = d.NJ, NG = d.NG, pitch = d.NJP;
    const int nvec = pitch / V;
    const int tid = threadIdx.x;
    const int m = t.trows;
    const int jv = tid % nvec, tr = tid / nvec < m ? tid / nvec : NI + 1;  // idle threads start past every row
    const int jb = jv * V;
    const int i0 = bx * t.TI;
    const int i1 = (bx == t.nrb - 1) ? NI : i0 + t.TI;
    const int rlo = i0 > 0 ? i0 - 1 : 0;
    const int c0 = 1 + by * t.GC;
    const int c1 = min(c0 + t.GC, NG - 1);
    const int step = d.counters[par];
    const bool y1_on = step + 1 >= d.pml_y_time;
    march_bookkeeping(d, par, step, bx == 0 && by == 0);

    // column data of this thread's vector, fixed for the whole march
    const Arr<R, VW> ayA = ldn<R, VW>(d.ayA + jb), ayP = ldn<R, VW>(d.ayP + jb);
    int yside = 0, ystore = 0;  // per element 2 bits: active y side; y1 / y2 storage
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
    const int ysm1 = jb >= 1 ? y_side(d, jb - 1, y1_on) : 0;  // column jb-1 (east face starting a vector)

    // shared memory: [ns mbarriers | 2 pressure slots | ring]
    unsigned char* smem = march_smem();
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    const int W = WIND ? 1 : 0;
    MarchGeo G;
    G.pitch = pitch;
    G.srows = t.rows_max + 1;
    G.rlo = rlo;
    G.ns = t.nstage;
    const int iclo = min(max(rlo, 1), NI - 2), ichi = min(max(i1 - 1, 1), NI - 2);
    G.r0[0] = iclo; G.nrow[0] = ichi + 2 - iclo;                              // u: i+1 for the pressure
    G.r0[1] = iclo; G.nrow[1] = ichi + 1 + W - iclo;                          // v
    G.r0[2] = iclo; G.nrow[2] = ichi + 1 + W - iclo;                          // w
    G.r0[3] = iclo - W; G.nrow[3] = ichi + 1 + W - iclo;                      // p: i-1 for the wind term
    {
        int off = 0;
        for (int f = 0; f < 4; ++f) {
            G.fb[f] = off - G.r0[f] * pitch;
            off += G.nrow[f] * pitch;
        }
        G.ss = off;
    }
    R* pb = reinterpret_cast<R*>(smem + 128);
    R* rg = pb + 2 * G.srows * pitch;
    const int first = c0 == 1 ? 1 : c0 - 1;  // first plane whose pressure is computed
    const int plo = first - W;                // first staged plane
    const R* const src[4] = {d.u_in, d.v_in, d.w_in, d.pold};
    // slab rows this block touches (stencil rows and their i-1 / i+1 neighbours)
    const int slo = max(rlo - 1, 0), shi = min(i1, NI - 1);

    if (tid == 0) {
        for (int s = 0; s < G.ns; ++s) mbar_init(&bar[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    auto issue = [&](int x) {  // producer: plane x into stage x % ns
        const int s = x % G.ns;
        fence_proxy_async();
        mbar_arrive_expect_tx(&bar[s], static_cast<uint32_t>(G.ss * sizeof(R)));
        R* dst = rg + static_cast<size_t>(s) * G.ss;
        for (int f = 0; f < 4; ++f)
            bulk_g2s(dst + G.fb[f] + G.r0[f] * pitch, src[f] + d.ix(x, G.r0[f], 0),
                     static_cast<uint32_t>(G.nrow[f] * pitch * sizeof(R)), &bar[s]);
    };
    // L2 prefetch of the PML slab rows of plane x (the slabs are read with
    // plain loads; the hint keeps those loads from waiting on DRAM)
    auto prefetch_slabs = [&](int x) {
        const int k = x - d.gOff;
        if (x < d.gOff || x >= NG) return;
        for (int s = 0; s < 6; ++s) {
            const Slab<R>& S = d.sl[s];
            if (!S.ni || (s == 2 && !y1_on) || !S.holds_k(k)) continue;
            const int a = max(slo, S.i0), b = min(shi, S.i0 + S.ni - 1);
            if (a > b) continue;
            const int q0 = S.q(a, S.ja, k);
            const uint32_t bytes = static_cast<uint32_t>((b - a + 1) * S.jp * sizeof(R));
            for (int c = 0; c < 4; ++c) bulk_prefetch_l2(S.rd[c] + q0, bytes);
        }
    };
    // A wait that runs out marks the block failed: that thread skips its
    // later waits, and once the issuing thread has failed it issues no more
    // copies, so every stage keeps at most one copy in flight for the drain
    // below (a stage is only refilled after its previous copy was seen).
    bool timed_out = false;
    const long long spin = d.wait_spin;
    auto wait_plane = [&](int x) {
        if (timed_out) return;
        if (!mbar_wait(&bar[x % G.ns], static_cast<uint32_t>(((x - plo) / G.ns) & 1), spin)) timed_out = true;
    };
    int issued_hi = plo - 1;
    if (tid == 0) {
        for (int x = plo; x <= min(plo + G.ns - 2, c1); ++x) {
            issue(x);
            issued_hi = x;
        }
        for (int x = first - 1; x <= first + 2; ++x) prefetch_slabs(x);
    }

    R bad = R(0);
    for (int q = first; q < c1; ++q) {
        const int slot = q & 1;
        if (tid == 0) {
            const int x = q + G.ns - 1 - W;  // into the stage plane q-1-W used last
            if (x <= c1 && x > issued_hi && !timed_out) {
                issue(x);
                issued_hi = x;
            }
            if (q + 3 <= c1) prefetch_slabs(q + 3);
        }
        if (q == first)
            for (int x = plo; x <= q + 1; ++x) wait_plane(x);
        else
            wait_plane(q + 1);
        const int oq = G.stage(q), on = G.stage(q + 1), om = WIND ? G.stage(q - 1) : 0;
        const PlaneC<R> pc = plane_c(d, q);
        const Arr<R, VW> ay = pc.pore ? ayP : ayA;
        const int ys = pc.pore ? 0 : yside;
        // phase 1: new pressure of rows rlo .. i1-1 at their clamped stencil rows
        for (int i = rlo + tr; i < i1; i += m) {
            const int ic = i < 1 ? 1 : (i > NI - 2 ? NI - 2 : i);
            const RowC<R> rc = row_c(d, pc, ic);
            stn<R, VW>(pb + G.prow(slot, i) + jb, march_p<R, WIND, VW, XF>(d, pc, rc, rg, G, oq, on, om, ic, jb, ay, ys));
        }
        __syncthreads();
        if (q == 1) {  // plane 0 (south face) pressure is plane 1's
            for (int i = rlo + tr; i < i1; i += m) stn<R, VW>(pb + G.prow(0, i) + jb, ldn<R, VW>(pb + G.prow(1, i) + jb));
            __syncthreads();
        }
        // phase 2: velocity, outputs, slabs, TDBC of rows i0 .. i1-1
        if (q >= c0)
            for (int i = i0 + tr; i < i1; i += m)
                march_emit<R, WIND, VW, XF>(d, pc, rg, pb, G, oq, on, slot, q, i, jb, ay, ys, ysm1, ystore, bad);
        __syncthreads();
    }
    if (!(bad == R(0))) atomicOr(d.status, 1);
    if (timed_out) {
        atomicOr(d.status, 2);
        if (tid == 0)  // let every copy this block issued land before the block exits
            for (int x = max(plo, issued_hi - G.ns + 1); x <= issued_hi; ++x)
                mbar_wait(&bar[x % G.ns], static_cast<uint32_t>(((x - plo) / G.ns) & 1));
    }
}

// XF: porous inclusions, the east TDBC, vectors with columns of both y
// layers and (east_scalar) an east column that starts a vector compiled in
// (the host picks the form without them for domains that have none: fewer
// registers and instructions)
template <typename R, bool WIND, int VW, bool XF>
__global__ void __launch_bounds__(256) k_march(__grid_constant__ const Dev<R> d, const MarchTiling t, int par) {
    march_block<R, WIND, VW, XF>(d, t, par, blockIdx.x, blockIdx.y);
}

// One block of a batched launch over independent domains (an ensemble of
// solves): block b runs row block bx, plane chunk by of domain `member`.
struct BatchWork {
    int member, bx, by;
};

// A domain of a batched launch: its fused-pass parameters at the parity of
// the step, that parity and its tile.
template <typename R>
struct BatchEntry {
    Dev<R> d;
    MarchTiling t;
    int par;
};

// entries [2][nmem]: phase 0 holds every member at the parity of the first
// step of the sequence, phase 1 at the other one; step s of a sequence
// passes phase s & 1.
template <typename R, bool WIND, int VW, bool XF>
__global__ void __launch_bounds__(256) k_march_batch(const BatchWork* __restrict__ work,
                                                     const BatchEntry<R>* __restrict__ entries, int nmem, int phase) {
    const BatchWork w = work[blockIdx.x];
    const BatchEntry<R>& e = entries[phase * nmem + w.member];
    march_block<R, WIND, VW, XF>(e.d, e.t, e.par, w.bx, w.by);
}

}  // namespace fdtd
