// Fused single-pass forward-backward step (FB_p_v): pressure and velocity
// of a plane in ONE marching pass over the unified g axis.
//
// Block = rows [i0, i1) of the i axis x all NJ columns x a chunk of "core"
// planes [c0, c1) within [1, NG-2]. The block marches g upward. For each
// plane it computes the new pressure of its rows plus one halo row below
// (i0-1) into shared memory (two plane slots: g and g-1), resolves the
// W/E pressure faces there, then computes the new velocity of its own rows
// from that shared-memory pressure (backward differences in i, j, g) -- so
// u, v, w, p are read once from HBM and written once, instead of the two
// passes' p round trip. Plane 0 (south face: porous or rigid ground) and
// plane NG-1 (north face) are copies of planes 1 and NG-2 (w = 0; east TDBC
// evaluated on the face row) and are emitted by the blocks owning planes 1
// and NG-2. The in-plane face walk is the same as the two-pass velocity
// kernel's; see fdtd_device.cuh.
//
// Two variants share the per-plane code:
//   k_fused      stencil inputs read straight from global memory
//   k_fused_tma  stencil inputs streamed into a shared-memory ring by 1D
//                bulk copies (cp.async.bulk, mbarrier transaction counts),
//                two planes ahead of the plane being computed
//
// Slab buffers: every read uses the values from before this step (Qp is
// advanced on the fly for the velocity stencil as Qp + dt * p, which is
// air::Update_PML_Qp, air.cpp:2388-2439), every write goes to the other
// buffer.
#pragma once

#include "fdtd_async.cuh"
#include "fdtd_device.cuh"

namespace fdtd {

struct FusedTiling {
    int TI;        // nominal rows per block (>= 2)
    int nrb;       // row blocks; the last one also takes the remainder rows
    int GC;        // core planes per block
    int nchunk;    // plane chunks
    int rows_max;  // most rows any block owns (shared-memory sizing)
    int nstage;    // bulk-copy ring depth (staged variant)
};

__device__ __forceinline__ unsigned char* fused_smem() {
    extern __shared__ __align__(16) unsigned char fdtd_smem[];
    return fdtd_smem;
}

// new-pressure planes in shared memory: two slots (g and g-1) x rows
// [rlo, rlo + srows) x NJ columns
template <typename R>
struct PlaneP {
    R* base;
    int srows, NJ, rlo;
    __device__ __forceinline__ R& operator()(int slot, int i, int j) const {
        return base[(static_cast<size_t>(slot) * srows + (i - rlo)) * NJ + j];
    }
};

// stencil inputs from the bulk-copy ring: stage (g % ns) holds rows
// [ra, ra + sr) of u, v, w, p of plane g, rows padded to the field pitch
template <typename R>
struct StagedFields {
    const R* base;
    int ns, sr, pitch, ra;
    __device__ __forceinline__ R at(int f, int i, int j, int g) const {
        return base[((static_cast<size_t>(g % ns) * 4 + f) * sr + (i - ra)) * pitch + j];
    }
    __device__ __forceinline__ R u(int i, int j, int g) const { return at(0, i, j, g); }
    __device__ __forceinline__ R v(int i, int j, int g) const { return at(1, i, j, g); }
    __device__ __forceinline__ R w(int i, int j, int g) const { return at(2, i, j, g); }
    __device__ __forceinline__ R p(int i, int j, int g) const { return at(3, i, j, g); }
};

template <typename R>
__device__ __forceinline__ void slab_update(const Dev<R>& d, int g, int i, int j, bool y1_on, const R* p,
                                            const R* u, const R* v, const R* w) {
    if (g < d.gOff) return;
    const int k = g - d.gOff;
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        const Slab<R>& S = d.sl[s];
        if (S.ni == 0 || (s == 2 && !y1_on)) continue;
        if (i < S.i0 || i >= S.i0 + S.ni || j < S.j0 || j >= S.j0 + S.nj || k < S.k0 || k >= S.k0 + S.nk) continue;
        const size_t q = S.at(i, j, k);
        if (p) S.wr[3][q] = S.rd[3][q] + d.dt * *p;
        if (u) {
            S.wr[0][q] = S.rd[0][q] + d.dt * *u;
            S.wr[1][q] = S.rd[1][q] + d.dt * *v;
            S.wr[2][q] = S.rd[2][q] + d.dt * *w;
        }
    }
}

template <typename R>
__device__ __forceinline__ void psi_update(const Dev<R>& d, int i, int k, double p) {
    const double vt = tdbc_v(d, i, k, p);
    const size_t o = (static_cast<size_t>(i) * d.Kair + k) * 6;
#pragma unroll
    for (int q = 0; q < 6; ++q) d.psi_out[o + q] = d.td_e[q] * d.psi_in[o + q] + d.td_adt[q] * vt;
}

// receivers (calculation_2D::get_pressure on p_n before the step) and the
// step counter: even steps read counters[0] and publish counters[1], odd
// steps the reverse (no block reads the word this launch writes)
template <typename R>
__device__ __forceinline__ void fused_step_bookkeeping(const Dev<R>& d, int par, int step) {
    if (blockIdx.x == 0 && blockIdx.y == 0) {
        const int tt = threadIdx.x;
        if (tt < d.nrec) {
            const long long n = d.rec_node[tt];
            double val = 0.0;
            if (n >= 0) val = static_cast<double>(d.pold[n]);
            if (fabs(val) < 1.0e-100) val = 0.0;
            d.rec_out[static_cast<size_t>(step) * d.nrec + tt] = val;
        }
        if (tt == 0) d.counters[par ^ 1] = step + 1;
    }
}

// phase 1: new pressure at the interior columns of rows rlo..i1-1 of plane gc
template <typename R, bool WIND, typename F>
__device__ __forceinline__ void fused_pressure(const Dev<R>& d, const F& f, const PlaneP<R>& P, int slot, int gc,
                                               int rlo, int i1, bool y1_on) {
    const int NI = d.NI, NJ = d.NJ;
    for (int i = rlo; i < i1; ++i) {
        const int ic = i < 1 ? 1 : (i > NI - 2 ? NI - 2 : i);
        for (int j = threadIdx.x; j < NJ; j += blockDim.x) {
            if (j == 0 || j == NJ - 1) continue;
            P(slot, i, j) = fresh_p<R, WIND>(d, f, ic, j, gc, y1_on);
        }
    }
}

// phase 2: west copy and east extrapolation (calculation_2D.cpp:650-672)
template <typename R>
__device__ __forceinline__ void fused_pressure_faces(const Dev<R>& d, const PlaneP<R>& P, int slot, int rlo, int i1) {
    const int NJ = d.NJ;
    const int ownE = (NJ - 1) % blockDim.x;
    for (int i = rlo; i < i1; ++i) {
        if (threadIdx.x == 0) P(slot, i, 0) = P(slot, i, 1);
        if (threadIdx.x == ownE)
            P(slot, i, NJ - 1) = R(15.0 / 8.0) * P(slot, i, NJ - 2) - R(5.0 / 4.0) * P(slot, i, NJ - 3) +
                                 R(3.0 / 8.0) * P(slot, i, NJ - 4);
    }
}

// phase 3: emit plane g (and the face plane 0 / NG-1 next to it): new
// pressure from shared memory, new velocity, slabs, TDBC state
template <typename R, bool WIND, typename F>
__device__ __forceinline__ void fused_emit(const Dev<R>& d, const F& f, const PlaneP<R>& P, int slot, int g, int i0,
                                           int i1, bool y1_on) {
    const int NI = d.NI, NJ = d.NJ, NG = d.NG;
    const bool pore = g < d.gAir0;
    for (int i = i0; i < i1; ++i) {
        for (int j = threadIdx.x; j < NJ; j += blockDim.x) {
            const R p = P(slot, i, j);
            const size_t c = d.ix(g, i, j);
            d.p_out[c] = p;
            if (!isfinite(static_cast<float>(p))) atomicOr(d.status, 1);
            slab_update<R>(d, g, i, j, y1_on, &p, nullptr, nullptr, nullptr);
            // velocity: in-plane faces B, F, W, E in reverse application order
            const bool onF = i == 0, onB = i == NI - 1, onW = j == 0, onE = j == NJ - 1;
            int ku = 0, kv = 0, ii = i, jj = j, ti = i;
            if (onB) { ku = 1; ii = NI - 2; }
            if (onF) { ku = 1; ii = 1; }
            if (onW) { kv = 1; jj = 1; }
            if (onE) {
                if (d.tdbc && !pore) { kv = 2; ti = ii; }
                else kv = 1;
                jj = NJ - 2;
            }
            const Vel3<R> fv = fresh_vel_core<R, WIND>(d, f, ii, jj, g, y1_on, P(slot, ii, jj), P(slot, ii - 1, jj),
                                                       P(slot, ii, jj - 1), P(slot ^ 1, ii, jj), true);
            const R u = ku == 0 ? fv.u : R(0);
            R v = kv == 0 ? fv.v : R(0);
            const R w = fv.w;
            if (kv == 2) v = static_cast<R>(tdbc_v(d, ti, g - d.gOff, static_cast<double>(P(slot, ti, NJ - 1))));
            d.u_out[c] = u;
            d.v_out[c] = v;
            d.w_out[c] = w;
            slab_update<R>(d, g, i, j, y1_on, nullptr, &u, &v, &w);
            if (d.tdbc && onE && g >= d.gOff) psi_update(d, i, g - d.gOff, static_cast<double>(P(slot, i, NJ - 1)));
            const R zero = R(0);
            if (g == 1) {  // south face plane: u, v of plane 1, w = 0
                const size_t c0i = d.ix(0, i, j);
                d.p_out[c0i] = p;
                d.u_out[c0i] = u;
                d.v_out[c0i] = v;
                d.w_out[c0i] = zero;
                slab_update<R>(d, 0, i, j, y1_on, &p, &u, &v, &zero);
                if (d.tdbc && onE && 0 >= d.gOff) psi_update(d, i, 0, static_cast<double>(P(slot, i, NJ - 1)));
            }
            if (g == NG - 2) {  // north face plane: u, v of plane NG-2 (east: TDBC on the face row), w = 0
                const size_t cti = d.ix(NG - 1, i, j);
                R vt = v;
                if (kv == 2)
                    vt = static_cast<R>(tdbc_v(d, ti, NG - 1 - d.gOff, static_cast<double>(P(slot, ti, NJ - 1))));
                d.p_out[cti] = p;
                d.u_out[cti] = u;
                d.v_out[cti] = vt;
                d.w_out[cti] = zero;
                slab_update<R>(d, NG - 1, i, j, y1_on, &p, &u, &vt, &zero);
                if (d.tdbc && onE) psi_update(d, i, NG - 1 - d.gOff, static_cast<double>(P(slot, i, NJ - 1)));
            }
        }
    }
}

template <typename R, bool WIND>
__global__ void __launch_bounds__(256) k_fused(__grid_constant__ const Dev<R> d, const FusedTiling t, int par) {
    const int NI = d.NI, NG = d.NG;
    const int i0 = blockIdx.x * t.TI;
    const int i1 = (blockIdx.x == t.nrb - 1) ? NI : i0 + t.TI;
    const int rlo = i0 > 0 ? i0 - 1 : 0;
    const int c0 = 1 + blockIdx.y * t.GC;
    const int c1 = min(c0 + t.GC, NG - 1);
    const int step = d.counters[par];
    const bool y1_on = step + 1 >= d.pml_y_time;
    fused_step_bookkeeping(d, par, step);
    const PlaneP<R> P{reinterpret_cast<R*>(fused_smem()), t.rows_max + 1, d.NJ, rlo};
    const GlobalFields<R> gf{d};
    for (int g = c0 - 1; g < c1; ++g) {
        const int slot = g & 1;
        const int gc = g == 0 ? 1 : g;  // plane 0 is the south face: copy of plane 1
        fused_pressure<R, WIND>(d, gf, P, slot, gc, rlo, i1, y1_on);
        __syncthreads();
        fused_pressure_faces(d, P, slot, rlo, i1);
        __syncthreads();
        if (g >= c0) fused_emit<R, WIND>(d, gf, P, slot, g, i0, i1, y1_on);
        __syncthreads();
    }
}

// Staged variant. Shared memory: [ns mbarriers | 2 pressure slots | ring of
// ns stages x 4 fields x sr rows x pitch]. Thread 0 is the producer: for
// plane x it arms barrier x % ns with the byte count and issues one bulk
// copy per field (the staged rows of one plane are contiguous in global
// memory). Every plane is waited for before use, by all threads, with a
// bounded wait; a timeout sets status bit 2, the block drains what it
// issued (bounded again) and the host reports the error.
template <typename R, bool WIND>
__global__ void __launch_bounds__(256) k_fused_tma(__grid_constant__ const Dev<R> d, const FusedTiling t, int par) {
    const int NI = d.NI, NJ = d.NJ, NG = d.NG, pitch = d.NJP;
    const int ns = t.nstage;
    const int i0 = blockIdx.x * t.TI;
    const int i1 = (blockIdx.x == t.nrb - 1) ? NI : i0 + t.TI;
    const int rlo = i0 > 0 ? i0 - 1 : 0;
    const int c0 = 1 + blockIdx.y * t.GC;
    const int c1 = min(c0 + t.GC, NG - 1);
    const int step = d.counters[par];
    const bool y1_on = step + 1 >= d.pml_y_time;
    fused_step_bookkeeping(d, par, step);

    unsigned char* smem = fused_smem();
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    const int srows = t.rows_max + 1;
    const int sr = t.rows_max + 3;
    R* pbase = reinterpret_cast<R*>(smem + 128);
    R* rbase = pbase + 2 * static_cast<size_t>(srows) * NJ;
    rbase = reinterpret_cast<R*>((reinterpret_cast<uintptr_t>(rbase) + 15) & ~uintptr_t(15));
    const PlaneP<R> P{pbase, srows, NJ, rlo};
    const int ra = rlo > 0 ? rlo - 1 : 0;
    const int rb = i1 < NI ? i1 : NI - 1;
    const int nr = rb - ra + 1;
    const StagedFields<R> sf{rbase, ns, sr, pitch, ra};
    const int W = WIND ? 1 : 0;
    const int first = c0 == 1 ? 1 : c0 - 1;  // first plane whose pressure is computed
    const int plo = first - W;                // first staged plane
    const uint32_t fbytes = static_cast<uint32_t>(nr) * pitch * sizeof(R);

    if (threadIdx.x == 0) {
        for (int s = 0; s < ns; ++s) mbar_init(&bar[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    auto issue = [&](int x) {  // producer: plane x into stage x % ns
        const int s = x % ns;
        fence_proxy_async();
        mbar_arrive_expect_tx(&bar[s], 4 * fbytes);
        const size_t off = d.ix(x, ra, 0);
        R* dst = rbase + (static_cast<size_t>(s) * 4 * sr) * pitch;
        const size_t fs = static_cast<size_t>(sr) * pitch;
        bulk_g2s(dst, d.u_in + off, fbytes, &bar[s]);
        bulk_g2s(dst + fs, d.v_in + off, fbytes, &bar[s]);
        bulk_g2s(dst + 2 * fs, d.w_in + off, fbytes, &bar[s]);
        bulk_g2s(dst + 3 * fs, d.pold + off, fbytes, &bar[s]);
    };
    bool timed_out = false;
    auto wait_plane = [&](int x) {
        if (!mbar_wait(&bar[x % ns], static_cast<uint32_t>(((x - plo) / ns) & 1))) timed_out = true;
    };
    int issued_hi = plo - 1;
    if (threadIdx.x == 0)
        for (int x = plo; x <= min(plo + ns - 2, c1); ++x) { issue(x); issued_hi = x; }

    for (int q = first; q < c1; ++q) {
        const int slot = q & 1;
        if (threadIdx.x == 0 && q + 2 <= c1 && q + 2 > issued_hi) { issue(q + 2); issued_hi = q + 2; }
        for (int x = q - W; x <= q + 1; ++x) wait_plane(x);
        fused_pressure<R, WIND>(d, sf, P, slot, q, rlo, i1, y1_on);
        __syncthreads();
        fused_pressure_faces(d, P, slot, rlo, i1);
        __syncthreads();
        if (q == 1) {  // plane 0 (south face) pressure is plane 1's
            for (int i = rlo; i < i1; ++i)
                for (int j = threadIdx.x; j < NJ; j += blockDim.x) P(slot ^ 1, i, j) = P(slot, i, j);
            __syncthreads();
        }
        if (q >= c0) fused_emit<R, WIND>(d, sf, P, slot, q, i0, i1, y1_on);
        __syncthreads();
    }
    if (timed_out) {
        atomicOr(d.status, 2);
        if (threadIdx.x == 0)  // let every copy this block issued land before the block exits
            for (int x = max(plo, issued_hi - ns + 1); x <= issued_hi; ++x)
                mbar_wait(&bar[x % ns], static_cast<uint32_t>(((x - plo) / ns) & 1));
    }
}

}  // namespace fdtd
