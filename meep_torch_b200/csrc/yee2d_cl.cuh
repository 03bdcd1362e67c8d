// Cluster-resident 2D TM steps for grids that fit in one thread-block cluster
// (sm_100a): the whole state of one structure stays on chip, spread over a cluster of
// up to 16 CTAs, for a ring's worth of steps (one launch per ring flush instead of
// one per step or per four steps).
//
// CTA r of the cluster owns rows [r R, r R + R); each of its threads owns one float4
// (a row, four columns) for the whole launch and keeps its Dz, Hx, Hy and 1/eps in
// registers. What a neighbour needs goes through shared memory: the Ez of every own
// row (EzS), the new Hx and Hy of every own row (HxS, HyS), the CPML memory of the
// layer cells; the rows next to another CTA travel as remote stores into that CTA's
// halo rows (distributed shared memory). A step is
//   H phase  Hx, Hy(n+1/2) of the own float4 (core/stepper_tm.py:85-128) from its Ez
//            and the neighbours' Ez (EzS: the right neighbour's first column, the row
//            below); magnetic sheet sources; H line / full-grid samples; Hx, Hy to HxS,
//            HyS (the last own row also to CTA r+1's halo row of HyS).
//   cluster barrier
//   D phase  Dz(n+1) (core/stepper_tm.py:130-166) from the own H and HyS (row above),
//            HxS (left column); electric source; Ez = Dz / eps to EzS (the first own row
//            also to CTA r-1's halo row of EzS) and the samples.
//   cluster barrier
// Each exchange row is written in one phase and read in the next, so the two barriers
// per step order every access. The state is read from the plan's buffer `par` at the
// start of the launch and written to `par ^ (nsub & 1)` at its end, preserving the
// plan's ping-pong parity. The arithmetic is the one-step tile kernel's, cell for cell
// (the results are bit-identical).
#pragma once

#include <cooperative_groups.h>

namespace mtb {

constexpr int CL_MAX = 16;                 // CTAs per cluster (non-portable size)
constexpr int CL_THREADS = 1024;           // one float4 per thread: R x pitch / 4 <= 1024

struct ClCtx {
    const mtb_yee2d_struct *structs;       // one cluster per structure
    const float *amp_e, *amp_h;            // coefficient rows of the first step [nsub][ncols]
    int ncols, nsub;
    float *ring;                           // ring slot of the first step
    int64_t slot_elems;
    int par;                               // buffer holding the old state
    int rows;                              // rows per CTA (R)
    int stage;                             // 1: line samples staged in shared memory
};

constexpr int CL_AMP = 1024;               // staged amplitudes per table (e, h)

// shared memory carve-up (bytes): structure copy, line samples, the launch's amplitude
// rows (e then h, CL_AMP floats each), profiles (H y b / a, E y b / a over pitch
// columns; H x b / a, E x b / a over R rows), then planes of pitch floats: EzS R + 1
// rows (row R: the halo row below), HyS R + 1 rows (row 0: the halo row above, row
// li + 1: own row li), HxS R rows, CPML memory psi 0..3 R rows each
constexpr size_t cl_align(size_t b) { return (b + 127) / 128 * 128; }
__host__ __device__ constexpr size_t cl_lines_off() { return cl_align(sizeof(mtb_yee2d_struct)); }
__host__ __device__ constexpr size_t cl_amp_off() {
    return cl_lines_off() + cl_align(sizeof(mtb_line_sample) * MAXL);
}
__host__ __device__ constexpr size_t cl_prof_off() { return cl_amp_off() + sizeof(float) * 2 * CL_AMP; }
__host__ __device__ constexpr size_t cl_planes_off(int rows, int pitch) {
    return cl_prof_off() + cl_align(sizeof(float) * 4 * ((size_t)pitch + rows));
}
__host__ __device__ constexpr size_t cl_smem(int rows, int pitch) {
    return cl_planes_off(rows, pitch) + sizeof(float) * (size_t)pitch * (7 * (size_t)rows + 2);
}
// line samples staged for the launch's steps after the planes: nsub x span floats,
// span = the extent of the structure's line offsets in a ring slot
__host__ __device__ constexpr size_t cl_smem_staged(int rows, int pitch, int64_t span, int nsub) {
    return cl_smem(rows, pitch) + sizeof(float) * (size_t)span * nsub;
}
// [lo, hi) of the line samples' ring offsets
__host__ __device__ inline void cl_line_span(const mtb_line_sample *L, int nl, int64_t &lo,
                                             int64_t &hi) {
    lo = nl > 0 ? L[0].ring_off : 0;
    hi = lo;
    for (int l = 0; l < nl; ++l) {
        lo = L[l].ring_off < lo ? L[l].ring_off : lo;
        const int64_t e = L[l].ring_off + (L[l].hi - L[l].lo);
        hi = e > hi ? e : hi;
    }
}

__device__ __forceinline__ void cl_ld4(const float *p, float (&v)[4]) {
    const float4 x = *reinterpret_cast<const float4 *>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void cl_st4(float *p, const float (&v)[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
// does a line sample of component comp cover a cell of row i, columns jb .. jb+3
__device__ __forceinline__ bool cl_hits(const mtb_line_sample *L, int nl, int comp, int i,
                                        int jb) {
    bool h = false;
    for (int l = 0; l < nl; ++l) {
        const mtb_line_sample &s = L[l];
        if (s.comp != comp) continue;
        if (s.kind == 0) h |= s.index == i && jb + 3 >= s.lo && jb < s.hi;
        else h |= i >= s.lo && i < s.hi && s.index >= jb && s.index < jb + 4;
    }
    return h;
}

// Split cluster barrier: the arrive releases this thread's shared-memory writes (own
// and remote), the wait acquires the other CTAs'. Global stores issued between the two
// (the ring samples) are not ordered by it, so they overlap the barrier instead of
// delaying its release.
__device__ __forceinline__ void cl_arrive() {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cl_wait() {
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(CL_THREADS, 1) k_cl_tm(const __grid_constant__ ClCtx C) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank(), ncl = (int)cl.num_blocks();
    const int sidx = blockIdx.x / ncl;
    extern __shared__ __align__(128) unsigned char cl_raw[];
    {
        const int *src = reinterpret_cast<const int *>(C.structs + sidx);
        int *dst = reinterpret_cast<int *>(cl_raw);
        for (int b = threadIdx.x; b < (int)(sizeof(mtb_yee2d_struct) / 4); b += CL_THREADS)
            dst[b] = src[b];
    }
    __syncthreads();
    const mtb_yee2d_struct &S = *reinterpret_cast<const mtb_yee2d_struct *>(cl_raw);
    const int nx = S.nx, ny = S.ny, P = S.pitch, R = C.rows;
    const int row0 = rank * R, nr = max(0, min(R, nx - row0));
    const int PL = R * P;
    mtb_line_sample *L = reinterpret_cast<mtb_line_sample *>(cl_raw + cl_lines_off());
    const int nl = S.n_lines;
    float *yHb = reinterpret_cast<float *>(cl_raw + cl_prof_off());
    float *yHa = yHb + P, *yEb = yHb + 2 * P, *yEa = yHb + 3 * P;
    float *xHb = yHb + 4 * P, *xHa = xHb + R, *xEb = xHb + 2 * R, *xEa = xHb + 3 * R;
    float *EzS = reinterpret_cast<float *>(cl_raw + cl_planes_off(R, P));
    float *HyS = EzS + (size_t)(R + 1) * P, *HxS = HyS + (size_t)(R + 1) * P;
    float *P0 = HxS + PL, *P1 = P0 + PL, *P2 = P1 + PL, *P3 = P2 + PL;
    // line samples and profiles as the tile kernels apply them ((1, 0) where a cell
    // is not updated or lies outside its layer)
    for (int l = threadIdx.x; l < nl; l += CL_THREADS) L[l] = S.lines[l];
    for (int j = threadIdx.x; j < P; j += CL_THREADS) {
        const bool oh = j <= ny - 2 && in_band(j, S.yband[0], S.yband[1]);
        const bool oe = j < ny && in_band(j, S.yband[2], S.yband[3]);
        yHb[j] = oh ? __ldg(S.hy_b + j) : 1.f;
        yHa[j] = oh ? __ldg(S.hy_a + j) : 0.f;
        yEb[j] = oe ? __ldg(S.ey_b + j) : 1.f;
        yEa[j] = oe ? __ldg(S.ey_a + j) : 0.f;
        EzS[(size_t)R * P + j] = 0.f;            // halo rows: zero at the grid's edges
        HyS[j] = 0.f;
    }
    for (int li = threadIdx.x; li < R; li += CL_THREADS) {
        const int i = row0 + li;
        const bool bxH = i <= nx - 2 && in_band(i, S.xband[0], S.xband[1]);
        const bool bxE = i >= 1 && i <= nx - 2 && in_band(i, S.xband[2], S.xband[3]);
        xHb[li] = bxH ? __ldg(S.hx_b + i) : 1.f;
        xHa[li] = bxH ? __ldg(S.hx_a + i) : 0.f;
        xEb[li] = bxE ? __ldg(S.ex_b + i) : 1.f;
        xEa[li] = bxE ? __ldg(S.ex_a + i) : 0.f;
    }
    // the source amplitudes of the launch's steps (from global memory when they do not fit;
    // read by plain loads, never __ldg, since they may sit in shared memory)
    const bool amp_smem = (int64_t)C.nsub * C.ncols <= CL_AMP;
    float *Ae = reinterpret_cast<float *>(cl_raw + cl_amp_off()), *Ah = Ae + CL_AMP;
    if (amp_smem)
        for (int e = threadIdx.x; e < C.nsub * C.ncols; e += CL_THREADS) {
            Ae[e] = C.amp_e[e];
            Ah[e] = C.amp_h[e];
        }
    // the neighbours' halo rows (same carve-up in every CTA): this CTA fills CTA r-1's
    // EzS row R and CTA r+1's HyS row 0
    const bool up = rank + 1 < ncl && row0 + R < nx, dn = rank > 0 && nr > 0;
    float *EzHalo = dn ? cl.map_shared_rank(EzS, rank - 1) + (size_t)R * P : EzS;
    float *HyHalo = up ? cl.map_shared_rank(HyS, rank + 1) : HyS;
    cl.sync();                                   // halo rows zeroed before any remote store

    // this thread's float4 and what it needs
    const int q4 = P / 4, items = nr * q4;
    const int it = threadIdx.x;
    const bool own = it < items;
    const int li = own ? it / q4 : 0, jb = own ? (it - li * q4) * 4 : 0, i = row0 + li;
    const int lo = li * P + jb;
    const uint32_t go = (uint32_t)i * P + jb;
    const bool hyRow = i <= nx - 2, dzRow = i >= 1 && i <= nx - 2;
    const bool bp0 = own && (in_band(jb, S.yband[0], S.yband[1]) ||
                             in_band(min(jb + 3, ny - 1), S.yband[0], S.yband[1]));
    const bool bp1 = own && hyRow && in_band(i, S.xband[0], S.xband[1]);
    const bool bp2 = own && dzRow && in_band(i, S.xband[2], S.xband[3]);
    const bool bp3 = own && (in_band(jb, S.yband[2], S.yband[3]) ||
                             in_band(min(jb + 3, ny - 1), S.yband[2], S.yband[3]));
    const bool sh2 = own && S.src_h2.n && i >= S.src_h2.row_lo && i <= S.src_h2.row_hi;
    const bool sh1 = own && hyRow && S.src_h1.n && i >= S.src_h1.row_lo && i <= S.src_h1.row_hi;
    const bool se = own && S.src_e.n && i >= S.src_e.row_lo && i <= S.src_e.row_hi;
    const bool lx = own && cl_hits(L, nl, MTB_C2_X, i, jb);
    const bool ly = own && cl_hits(L, nl, MTB_C2_Y, i, jb);
    const bool lm = own && cl_hits(L, nl, MTB_C2_MAIN, i, jb);
    const bool fx = own && S.ring_full[1] >= 0, fy = own && S.ring_full[2] >= 0;
    const bool fm = own && S.ring_full[0] >= 0;
    // staged line samples: step s, ring offset o at stage[s * span + o - slo]
    int64_t slo = 0, shi = 0;
    cl_line_span(L, nl, slo, shi);
    const int span = (int)(shi - slo);
    float *stage = P3 + PL;
    const int par = C.par;
    float dz[4], hx[4], hy[4], ie[4];
    zero4(dz); zero4(hx); zero4(hy); zero4(ie);
    if (own) {
        cl_ld4(S.f_main[par] + go, dz);
        cl_ld4(S.f_x[par] + go, hx);
        cl_ld4(S.f_y[par] + go, hy);
        cl_ld4(S.inv_eps_a + go, ie);
        float v[4];
        cl_ld4(S.psi[0][par] + go, v); cl_st4(P0 + lo, v);
        cl_ld4(S.psi[1][par] + go, v); cl_st4(P1 + lo, v);
        cl_ld4(S.psi[2][par] + go, v); cl_st4(P2 + lo, v);
        cl_ld4(S.psi[3][par] + go, v); cl_st4(P3 + lo, v);
        float ez[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) ez[q] = dz[q] * ie[q];
        cl_st4(EzS + lo, ez);
        if (li == 0 && dn) cl_st4(EzHalo + jb, ez);
        cl_st4(HyS + lo + P, hy);
        if (li == R - 1 && up) cl_st4(HyHalo + jb, hy);
    }
    cl.sync();                                   // every CTA's state is in place

    const float dt = S.dt, rdx = 1.0f / S.dx;
    for (int s = 0; s < C.nsub; ++s) {
        const float *ae = (amp_smem ? Ae : C.amp_e) + (size_t)s * C.ncols;
        const float *ah = (amp_smem ? Ah : C.amp_h) + (size_t)s * C.ncols;
        float *ring = C.ring + (size_t)s * C.slot_elems;
        float *lring = C.stage ? stage + (int64_t)s * span - slo : ring;   // line samples
        // ---- H(n+1/2): core/stepper_tm.py:85-128
        if (own) {
            float ez1[4], ez2[4], p0[4], p1[4], hyb[4], hya[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) ez1[q] = dz[q] * ie[q];
            const float ezR = (jb + 4 < P) ? EzS[lo + 4] : 0.f;
            if (li + 1 < nr || up) cl_ld4(EzS + lo + P, ez2);   // row below / halo row
            else zero4(ez2);
            if (bp0) cl_ld4(P0 + lo, p0); else zero4(p0);
            if (bp1) cl_ld4(P1 + lo, p1); else zero4(p1);
            cl_ld4(yHb + jb, hyb); cl_ld4(yHa + jb, hya);
            // Hx row i: valid j <= ny-2
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const bool vH = jb + q <= ny - 2;
                const float er = (q < 3) ? ez1[q + 1] : ezR;
                const float d = (er - ez1[q]) * rdx;
                const float pv = hyb[q] * p0[q] + hya[q] * d;
                const float hn = hx[q] - dt * (d + pv);
                hx[q] = vH ? hn : hx[q];
                p0[q] = vH ? pv : p0[q];
            }
            if (sh2) apply_cells_a(S.src_h2, i, ah[S.src_h2.amp_col], jb, hx);
            // Hy row i: valid i <= nx-2
            {
                const float b = xHb[li], a = xHa[li];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float d = (ez2[q] - ez1[q]) * rdx;
                    const float pv = b * p1[q] + a * d;
                    const float hn = hy[q] + dt * (d + pv);
                    hy[q] = hyRow ? hn : hy[q];
                    p1[q] = hyRow ? pv : p1[q];
                }
                if (sh1) apply_cells_a(S.src_h1, i, ah[S.src_h1.amp_col], jb, hy);
            }
            cl_st4(HxS + lo, hx);
            cl_st4(HyS + lo + P, hy);
            if (li == R - 1 && up) cl_st4(HyHalo + jb, hy);
            if (bp0) cl_st4(P0 + lo, p0);
            if (bp1) cl_st4(P1 + lo, p1);
        }
        cl_arrive();
        if (own) {
            if (fx) cl_st4(ring + S.ring_full[1] + go, hx);
            if (fy) cl_st4(ring + S.ring_full[2] + go, hy);
            if (lx) sample_row(L, nl, MTB_C2_X, i, jb, true, hx, lring);
            if (ly) sample_row(L, nl, MTB_C2_Y, i, jb, true, hy, lring);
        }
        cl_wait();
        // ---- Dz(n+1), source, Ez = Dz / eps: core/stepper_tm.py:130-166, :221-231
        float ez[4];
        if (own) {
            float hyP[4], p2[4], p3[4], eyb[4], eya[4];
            cl_ld4(HyS + lo, hyP);                               // row above / halo row
            const float hxm0 = (jb >= 1) ? HxS[lo - 1] : 0.f;
            if (bp2) cl_ld4(P2 + lo, p2); else zero4(p2);
            if (bp3) cl_ld4(P3 + lo, p3); else zero4(p3);
            cl_ld4(yEb + jb, eyb); cl_ld4(yEa + jb, eya);
            const float exb = xEb[li], exa = xEa[li];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j = jb + q;
                const bool vD = dzRow && j >= 1 && j <= ny - 2;
                const float hxm = (q == 0) ? hxm0 : hx[q - 1];
                const float dhy = (hy[q] - hyP[q]) * rdx;
                const float dhx = (hx[q] - hxm) * rdx;
                const float q2 = exb * p2[q] + exa * dhy;
                const float q3 = eyb[q] * p3[q] + eya[q] * dhx;
                const float curl = (dhy + q2) - (dhx + q3);
                const float dnv = dz[q] + dt * curl;
                dz[q] = vD ? dnv : dz[q];
                p2[q] = vD ? q2 : p2[q];
                p3[q] = vD ? q3 : p3[q];
            }
            if (se) apply_cells_a(S.src_e, i, ae[S.src_e.amp_col], jb, dz);
#pragma unroll
            for (int q = 0; q < 4; ++q) ez[q] = dz[q] * ie[q];
            cl_st4(EzS + lo, ez);
            if (li == 0 && dn) cl_st4(EzHalo + jb, ez);
            if (bp2) cl_st4(P2 + lo, p2);
            if (bp3) cl_st4(P3 + lo, p3);
        }
        cl_arrive();
        if (own) {
            if (fm) cl_st4(ring + S.ring_full[0] + go, ez);
            if (lm) sample_row(L, nl, MTB_C2_MAIN, i, jb, true, ez, lring);
        }
        cl_wait();
    }
    // ---- the staged line samples of the own rows to the ring (the last phase wrote its
    // samples after the cluster arrive, so the CTA synchronises once more first)
    __syncthreads();
    if (C.stage) {
        for (int l = 0; l < nl; ++l) {
            const mtb_line_sample &ln = L[l];
            int k0, k1;                              // own part of the line, as p = k - lo
            if (ln.kind == 0) {
                const bool mine = ln.index >= row0 && ln.index < row0 + nr;
                k0 = 0;
                k1 = mine ? ln.hi - ln.lo : 0;
            } else {
                k0 = max(ln.lo, row0) - ln.lo;
                k1 = min(ln.hi, row0 + nr) - ln.lo;
            }
            const int len = k1 - k0;
            for (int e = threadIdx.x; e < len * C.nsub; e += CL_THREADS) {
                const int s = e / len, k = k0 + (e - s * len);
                C.ring[(size_t)s * C.slot_elems + ln.ring_off + k] =
                    stage[(int64_t)s * span + ln.ring_off - slo + k];
            }
        }
    }
    // ---- the state to the buffer the plan reads next
    if (own) {
        const int pw = par ^ (C.nsub & 1);
        float v[4];
        cl_st4(S.f_main[pw] + go, dz);
        cl_st4(S.f_x[pw] + go, hx);
        cl_st4(S.f_y[pw] + go, hy);
        cl_ld4(P0 + lo, v); cl_st4(S.psi[0][pw] + go, v);
        cl_ld4(P1 + lo, v); cl_st4(S.psi[1][pw] + go, v);
        cl_ld4(P2 + lo, v); cl_st4(S.psi[2][pw] + go, v);
        cl_ld4(P3 + lo, v); cl_st4(S.psi[3][pw] + go, v);
    }
}

}  // namespace mtb
