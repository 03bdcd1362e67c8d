// One-pass 3D Yee step (H then E of the same x plane in one kernel) for sm_100a:
// the functional stepper's CPML path, core/stepper_3d.py:363-445, and its soft
// source, :448-482, with the arithmetic of the split kernels k_yee3d_h /
// k_yee3d_e cell for cell (the results are bit-identical to theirs).
//
// Work: the y axis is cut into tiles of at most TY rows (tile t: rows ytab[t] ..
// ytab[t+1]-1); (tile, x plane) pairs are numbered tile-major and every block of a
// persistent grid takes one contiguous share of that sequence. The host cuts
// tile-major shares of equal estimated cost (a pair in an x or y CPML layer costs
// more) or, when asked, lockstep shares (every tile split at the same x planes, one
// share per block, tile heights balanced by cost) so that y-neighbour tiles pass a
// plane at about the same time and the halo rows one reads are still in L2.
// Within a segment the block marches along x. Per x plane p:
//   H phase  H(n+1/2) of plane p for the tile's rows and the row below it (that
//            halo row is recomputed, never stored) from staged E(n) of planes p
//            and p+1, staged H(n-1/2) and z-layer CPML memory; the new H goes to
//            HBM and its Hx / Hz (and the Hy of each z half's last column) to a
//            shared exchange plane (double buffered).
//   barrier  (one per plane)
//   E phase  E(n+1) of plane p for the tile's rows from the new H of the cell and
//            of its y-1 / z-1 neighbours (exchange plane), H(n+1/2) of plane
//            p-1 (kept in registers from the previous plane), staged eps of planes p
//            and p+1; soft current cells; E(n+1) to HBM.
// A segment starting at x = xs > 0 first recomputes H of plane xs-1 (registers
// only). Every evolving array is a ping-pong pair, so the recomputation reads the
// same old values as the neighbouring segment.
//
// Staging: per x plane, TMA 3D tensor copies (cp.async.bulk.tensor.3d; rows and
// planes outside the grid read as zero) bring E(n) (rows y0-1 .. y0+TY), eps (rows
// y0 .. y0+TY), H(n-1/2) (rows y0-1 .. y0+TY-1) and, where the z axis has CPML
// layers, the z-layer CPML memory of both sides (two XM_BZ-wide boxes per array)
// into one of XM_NS stages, completion counted on the stage's mbarrier. The stage
// of plane m is refilled with plane m + XM_NS once every thread is past the
// barrier of plane m + 1, so each copy has a plane of compute to land. The x- and
// y-layer CPML memory (whole planes / tiles, a minority of the elements) is read
// from HBM in the element. Every wait is bounded by %globaltimer: an expired wait
// raises the plan's error flag, the block finishes its sequence (results invalid,
// reported by the host), and exits only after its copies in flight have landed or a
// second bounded wait expired.
//
// Threads: warp w owns row slot w / V (slot 0 = row y0-1, slot r = row y0-1+r)
// and z columns (w % V) * 128 + 4 lane .. +3, one float4 of each array.
#pragma once

namespace mtb {

constexpr int XM_NS = 4;                               // staged x planes
constexpr int XM_BZ = 24;                              // z-layer box width (floats)
constexpr unsigned long long XM_WAIT_NS = 2000000000ull;  // bounded wait: 2 s

struct XmMaps {
    CUtensorMap e[2][3];   // E of buffer 0 / 1: box 128V z x (TY+2) rows x 1 plane
    CUtensorMap h[2][3];   // H of buffer 0 / 1: box 128V z x (TY+1) rows x 1 plane
    CUtensorMap pz[2][4];  // psi 1, 2 (H side), 7, 8 (E side): box XM_BZ x (TY+1) x 1
    CUtensorMap eps;       // box 128V z x (TY+1) rows x 1 plane
    int zl, zh;            // z-layer boxes [0, XM_BZ) and [zh, zh + XM_BZ): a float4
                           // of z-layer cells lies below zl or at / above zh
    int npz;               // 1: the z-layer boxes are staged
    const float *ptab;     // profiles masked as the kernels apply them, (1, 0) outside the
                           // layers: x [H b, H a, E b, E a][nx], y [..][ny], z [..][zpitch]
    const int *ytab;       // first row of each tile, tiles + 1 entries (last = ny)
};

template <int V, int TY>
struct XmShape {
    static constexpr int ZB = 128 * V;                 // staged z extent
    static constexpr int SLOTS = TY + 1;               // row slots (slot 0: halo row)
    static constexpr int THREADS = 32 * V * SLOTS;
    static constexpr int EROWS = TY + 2;               // E rows y0-1 .. y0+TY
    static constexpr int PROWS = TY + 1;               // eps rows y0 .. y0+TY
    static constexpr int PZB = (SLOTS * XM_BZ + 31) / 32 * 32;   // one z-layer box, padded
    // stage carve-up (floats): Ex Ey Ez | eps | Hx Hy Hz | psi 1 2 7 8 x (low, high)
    static constexpr int OFF_EPS = 3 * EROWS * ZB;
    static constexpr int OFF_H = OFF_EPS + PROWS * ZB;
    static constexpr int OFF_PZ = OFF_H + 3 * SLOTS * ZB;
    static constexpr int STAGE = OFF_PZ + 8 * PZB;
    static constexpr uint32_t BYTES_BASE = (uint32_t)OFF_PZ * 4;
    static constexpr uint32_t BYTES_PZ = 8u * SLOTS * XM_BZ * 4;
    // exchange buffer: Hx, Hz rows, then the Hy of each z half's last column
    static constexpr int XH = 2 * SLOTS * ZB + 4 * SLOTS;
    static constexpr size_t SMEM = sizeof(float) * ((size_t)XM_NS * STAGE + 2 * XH) +
                                   XM_NS * sizeof(uint64_t);
};

__device__ __forceinline__ uint32_t xm_s32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long xm_clock() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool xm_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(xm_s32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// Bounded wait for one stage; false once the limit passed (the error flag is set).
__device__ __forceinline__ bool xm_wait(uint64_t *bar, uint32_t parity, int *err) {
    if (xm_try(bar, parity)) return true;
    const unsigned long long t0 = xm_clock();
    while (!xm_try(bar, parity)) {
        if (xm_clock() - t0 > XM_WAIT_NS) {
            atomicExch(err, 1);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void xm_tma3(float *dst, const CUtensorMap *map, int z, int y, int x,
                                        uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(xm_s32(dst)), "l"(map), "r"(z), "r"(y), "r"(x), "r"(xm_s32(bar)) : "memory");
}

// The block's share of the (tile, plane) sequence and its segments. Elements of
// tile t: plane xs-1 (halo, when xs > 0), the body xs .. xe-1, plane xe (tail,
// staged only as the E(p+1) of the last body plane, when xe < nx).
struct XmSeq {
    int t0, t1;            // first and last tile
    int xs0, xe1;          // body start in tile t0, body end in tile t1
    int nx;
    __device__ void init(int64_t u0, int64_t u1, int nx_) {
        nx = nx_;
        t0 = (int)(u0 / nx_);
        t1 = (int)((u1 - 1) / nx_);
        xs0 = (int)(u0 - (int64_t)t0 * nx_);
        xe1 = (int)(u1 - (int64_t)t1 * nx_);
    }
    __device__ int xs(int t) const { return t == t0 ? xs0 : 0; }
    __device__ int xe(int t) const { return t == t1 ? xe1 : nx; }
    __device__ int first(int t) const { const int s = xs(t); return s > 0 ? s - 1 : 0; }
    __device__ int last(int t) const { const int e = xe(t); return e < nx ? e : nx - 1; }
    // advance (t, p) to the next element; false past the end
    __device__ bool next(int &t, int &p) const {
        if (p < last(t)) { ++p; return true; }
        if (t >= t1) return false;
        ++t;
        p = first(t);
        return true;
    }
};

template <int V, int TY>
__device__ __forceinline__ void xm_issue(const XmMaps &M, int par, int t, int p, float *stage,
                                         uint64_t *bar) {
    using S = XmShape<V, TY>;
    const int y0 = __ldg(M.ytab + t);
    const uint32_t bytes = S::BYTES_BASE + (M.npz ? S::BYTES_PZ : 0u);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 ::"r"(xm_s32(bar)), "r"(bytes) : "memory");
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        xm_tma3(stage + c * S::EROWS * S::ZB, &M.e[par][c], 0, y0 - 1, p, bar);
        xm_tma3(stage + S::OFF_H + c * S::SLOTS * S::ZB, &M.h[par][c], 0, y0 - 1, p, bar);
    }
    xm_tma3(stage + S::OFF_EPS, &M.eps, 0, y0, p, bar);
    if (M.npz) {
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            xm_tma3(stage + S::OFF_PZ + (2 * a) * S::PZB, &M.pz[par][a], 0, y0 - 1, p, bar);
            xm_tma3(stage + S::OFF_PZ + (2 * a + 1) * S::PZB, &M.pz[par][a], M.zh, y0 - 1, p, bar);
        }
    }
}

// L2 prefetch (cp.async.bulk.prefetch) of the x / y layer CPML memory an element will
// read: the rows y0-1 .. y1-1 of plane p are one contiguous run per array.
__device__ __forceinline__ void xm_l2_psi(const Split3 &P, const XmMaps &M, int t, int p) {
    const int ny = P.ny, y0 = __ldg(M.ytab + t);
    const int r0 = max(y0 - 1, 0), r1 = min(__ldg(M.ytab + t + 1), ny);
    const bool xb = inband(P.B, 0, 0, p) || inband(P.B, 0, 1, p);
    bool yb = false;
    for (int r = r0; r < r1; ++r) yb |= inband(P.B, 1, 0, r) || inband(P.B, 1, 1, r);
    if (!xb && !yb) return;
    const size_t off = ((size_t)p * ny + r0) * P.zp;
    const uint32_t bytes = (uint32_t)(r1 - r0) * P.zp * 4;
    const int ya[4] = {0, 5, 6, 11}, xa[4] = {3, 4, 9, 10};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (yb)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                         ::"l"(P.pi[ya[q]] + off), "r"(bytes) : "memory");
        if (xb)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                         ::"l"(P.pi[xa[q]] + off), "r"(bytes) : "memory");
    }
}

__device__ __forceinline__ void lds4v(const float *p, float (&v)[4]) {
    const float4 x = *reinterpret_cast<const float4 *>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}

// Per-thread state of the march, shared by the element bodies.
struct XmCtx {
    float *stages, *xh;                // stage ring, exchange planes (shared)
    uint64_t *bars;
    int tid, lane, slot, zw, kb, pzo;
    int ready, issued, pt, pp;         // stage waits done; producer (thread 0) cursor
    bool ok, pmore;
    float hyp[4], hzp[4];              // H(n+1/2) of the previous plane (own cell)
    float zp[4][4];                    // masked z profiles of the own cells: H b, H a, E b, E a
};

// One element (plane p of tile t). XY: the plane or the row lies in an x or y CPML
// layer (warp-uniform); otherwise the x / y layer terms, whose memory and profile
// are identically (0; 1, 0) there, are left out.
template <int V, int TY, bool XY>
__device__ __forceinline__ void xm_elem(const Split3 &P, const XmMaps &M, const XmSeq &Q,
                                        XmCtx &c, int n, int t, int p, bool halo, bool tail,
                                        bool has_next, const float *__restrict__ amp, int par,
                                        int *__restrict__ err) {
    using S = XmShape<V, TY>;
    constexpr int ZB = S::ZB, ER = S::EROWS;
    const int nx = P.nx, ny = P.ny, nz = P.nz, ZP = P.zp;
    const int lane = c.lane, slot = c.slot, kb = c.kb;
    const float dt = P.dt, rdx = P.rdx;
    const int j = __ldg(M.ytab + t) - 1 + slot, i = p;
    // rows past the tile (a tile shorter than TY) are the next tile's: not stored
    const int jend = min(__ldg(M.ytab + t + 1), ny);
    const bool act = j >= 0 && j < jend && kb < ZP;
    const uint32_t g = (uint32_t)i * ((uint32_t)ny * ZP) + (uint32_t)(max(j, 0) * ZP + kb);
    const bool xok = i <= nx - 2, vyH = j <= ny - 2;
    const bool bx = XY && act && xok && inband(P.B, 0, 0, i);
    const bool by = XY && act && vyH && inband(P.B, 1, 0, j);
    bool bz = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) bz |= act && kb + q <= nz - 2 && inband(P.B, 2, 0, kb + q);
    const float *xt = M.ptab, *yt = M.ptab + 4 * nx;      // masked x / y profiles
    // E phase of this warp (warp-uniform) and its flags
    const bool eact = !tail && !halo && slot > 0 && j < jend;
    const bool iin = i >= 1 && i <= nx - 2, jin = j >= 1 && j <= ny - 2;
    const bool pmx = P.pmc & 1, pmy = (P.pmc >> 1) & 1, pmz = (P.pmc >> 2) & 1;
    const bool bxe = XY && eact && act && iin && inband(P.B, 0, 1, i);
    const bool bye = XY && eact && act && jin && inband(P.B, 1, 1, j);
    // x / y layer memory (band planes / tiles only) and the row's soft current cells
    // from HBM / L2, issued before the stage wait so that the H phase covers them
    float p0[4], p3[4], p4[4], p5[4], p6[4], p9[4], p10[4], p11[4];
    z4(p0); z4(p3); z4(p4); z4(p5); z4(p6); z4(p9); z4(p10); z4(p11);
    if (XY && !tail) {
        if (by) ld4v(P.pi[0] + g, p0);
        if (bx) ld4v(P.pi[3] + g, p3);
        if (vyH && bx) ld4v(P.pi[4] + g, p4);
        if (xok && by) ld4v(P.pi[5] + g, p5);
        if (xok && bye) ld4v(P.pi[6] + g, p6);
        if (vyH && bxe) ld4v(P.pi[9] + g, p9);
        if (bxe) ld4v(P.pi[10] + g, p10);
        if (bye) ld4v(P.pi[11] + g, p11);
    }
    int e0 = 0, e1x = 0;
    if (eact && act && P.src_n > 0) {
        e0 = __ldg(P.src_row + i * ny + j);
        e1x = __ldg(P.src_row + i * ny + j + 1);
    }
    // ---- stages of planes p and p+1
    const int need = n + (has_next ? 2 : 1);
    while (c.ready < need) {
        if (c.ok) c.ok = xm_wait(c.bars + c.ready % XM_NS, (c.ready / XM_NS) & 1, err);
        ++c.ready;
    }
    const float *st = c.stages + (n % XM_NS) * S::STAGE;
    const float *sn = c.stages + ((n + 1) % XM_NS) * S::STAGE;
    const float *Ex = st, *Ey = st + ER * ZB, *Ez = st + 2 * ER * ZB, *Ep = st + S::OFF_EPS;
    const float *pz = st + S::OFF_PZ + c.pzo;
    float *xw = c.xh + (n & 1) * S::XH;
    float hx[4], hy[4], hz[4];
    z4(hx); z4(hy); z4(hz);
    if (!tail) {
        // ---- H(n+1/2) of (i, j): core/stepper_3d.py:367-393
        float ex[4], ey[4], ez[4], ezj[4], exj[4], ezi[4], eyi[4], p1[4], p2[4], hzb[4], hza[4];
        const int r = slot * ZB + kb;
        lds4v(Ex + r, ex); lds4v(Ey + r, ey); lds4v(Ez + r, ez);
        lds4v(Ez + r + ZB, ezj); lds4v(Ex + r + ZB, exj);
        lds4v(st + S::OFF_H + r, hx);
        lds4v(st + S::OFF_H + S::SLOTS * ZB + r, hy);
        lds4v(st + S::OFF_H + 2 * S::SLOTS * ZB + r, hz);
        if (has_next) {
            lds4v(sn + ER * ZB + r, eyi);
            lds4v(sn + 2 * ER * ZB + r, ezi);
        } else {
            z4(eyi); z4(ezi);
        }
        z4(p1); z4(p2);
        if (vyH && bz) lds4v(pz, p1);
        if (xok && bz) lds4v(pz + 2 * S::PZB, p2);
#pragma unroll
        for (int q = 0; q < 4; ++q) { hzb[q] = c.zp[0][q]; hza[q] = c.zp[1][q]; }
        float eyk = 0.f, exk = 0.f;
        if (lane == 31 && kb + 4 < ZP) { eyk = Ey[r + 4]; exk = Ex[r + 4]; }
        float hxb = 1.f, hxa = 0.f, hyb = 1.f, hya = 0.f;
        if (XY) {
            hxb = __ldg(xt + i); hxa = __ldg(xt + nx + i);
            const int jc = min(max(j, 0), ny - 1);
            hyb = __ldg(yt + jc); hya = __ldg(yt + ny + jc);
        }
        {
            const float t0 = __shfl_down_sync(0xffffffffu, ey[0], 1);
            const float t1 = __shfl_down_sync(0xffffffffu, ex[0], 1);
            if (lane != 31) { eyk = t0; exk = t1; }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const bool vz = kb + q <= nz - 2, vzE = kb + q < nz;
            const float eyn = (q < 3) ? ey[q + 1] : eyk;
            const float exn = (q < 3) ? ex[q + 1] : exk;
            // x / y terms: d + (b psi + a d), which is d itself outside those layers
            {
                float qy = 0.f, qz;
                const float dy = y3_d(ezj[q], ez[q], rdx);
                const float cu = __fsub_rn(XY ? y3_s(dy, hyb, hya, p0[q], qy) : dy,
                                           y3_s(y3_d(eyn, ey[q], rdx), hzb[q], hza[q], p1[q], qz));
                const bool v = vyH && vz;
                const float hn = y3_h(hx[q], cu, dt);
                hx[q] = v ? hn : hx[q];
                if (XY) p0[q] = v ? qy : p0[q];
                p1[q] = v ? qz : p1[q];
            }
            {
                float qz, qx = 0.f;
                const float dx = y3_d(ezi[q], ez[q], rdx);
                const float cu = __fsub_rn(y3_s(y3_d(exn, ex[q], rdx), hzb[q], hza[q], p2[q], qz),
                                           XY ? y3_s(dx, hxb, hxa, p3[q], qx) : dx);
                const bool v = xok && vz;
                const float hn = y3_h(hy[q], cu, dt);
                hy[q] = v ? hn : hy[q];
                p2[q] = v ? qz : p2[q];
                if (XY) p3[q] = v ? qx : p3[q];
            }
            {
                float qx = 0.f, qy = 0.f;
                const float dx = y3_d(eyi[q], ey[q], rdx), dy = y3_d(exj[q], ex[q], rdx);
                const float cu = XY ? __fsub_rn(y3_s(dx, hxb, hxa, p4[q], qx),
                                                y3_s(dy, hyb, hya, p5[q], qy))
                                    : __fsub_rn(dx, dy);
                const bool v = xok && vyH && vzE;
                const float hn = y3_h(hz[q], cu, dt);
                hz[q] = v ? hn : hz[q];
                if (XY) {
                    p4[q] = v ? qx : p4[q];
                    p5[q] = v ? qy : p5[q];
                }
            }
        }
        if (!act) { z4(hx); z4(hy); z4(hz); }
        if (!halo) {
            const int o = slot * ZB + kb;
            st4v(xw + o, hx);
            st4v(xw + S::SLOTS * ZB + o, hz);
            if (lane == 31) xw[2 * S::SLOTS * ZB + 4 * slot + c.zw] = hy[3];
            if (act && slot > 0) {
                st4v(P.ho[0] + g, hx);
                st4v(P.ho[1] + g, hy);
                st4v(P.ho[2] + g, hz);
                if (vyH && bz) st4v(P.po[1] + g, p1);
                if (xok && bz) st4v(P.po[2] + g, p2);
                if (XY) {
                    if (by) st4v(P.po[0] + g, p0);
                    if (bx) st4v(P.po[3] + g, p3);
                    if (vyH && bx) st4v(P.po[4] + g, p4);
                    if (xok && by) st4v(P.po[5] + g, p5);
                }
            }
        }
    }
    __syncthreads();
    // stage of element n-1 is free: stage element n + XM_NS - 1 there
    if (c.tid == 0 && c.pmore && c.issued == n + XM_NS - 1) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const int s = c.issued % XM_NS;
        xm_issue<V, TY>(M, par, c.pt, c.pp, c.stages + s * S::STAGE, c.bars + s);
        ++c.issued;
        c.pmore = Q.next(c.pt, c.pp);
        // x / y layer memory of the element after next into L2
        int t2 = t, p2 = p;
        if (Q.next(t2, p2) && Q.next(t2, p2)) xm_l2_psi(P, M, t2, p2);
    }
    if (eact) {
        // ---- E(n+1) of (i, j): core/stepper_3d.py:395-437, source :448-482
        bool bze = false;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = kb + q;
            bze |= act && k >= 1 && k <= nz - 2 && inband(P.B, 2, 1, k);
        }
        float p7[4], p8[4];
        z4(p7); z4(p8);
        if (xok && bze) lds4v(pz + 4 * S::PZB, p7);
        if (vyH && bze) lds4v(pz + 6 * S::PZB, p8);
        const int o = slot * ZB + kb;
        const float *xr = c.xh + (n & 1) * S::XH;
        float hzm[4], hxm[4], ep[4], epj[4], epi[4], en[3][4], ezb[4], eza[4];
        lds4v(xr + S::SLOTS * ZB + o - ZB, hzm);
        lds4v(xr + o - ZB, hxm);
        const int re = (slot - 1) * ZB + kb;           // eps row of j
        lds4v(Ep + re, ep);
        if (j + 1 < ny) lds4v(Ep + re + ZB, epj); else one4(epj);
        if (has_next) lds4v(sn + S::OFF_EPS + re, epi); else one4(epi);
        lds4v(Ex + o, en[0]); lds4v(Ey + o, en[1]); lds4v(Ez + o, en[2]);
#pragma unroll
        for (int q = 0; q < 4; ++q) { ezb[q] = c.zp[2][q]; eza[q] = c.zp[3][q]; }
        float hyk = 0.f, hxk = 0.f, epk = 1.f;
        if (lane == 0 && kb >= 1) {
            hyk = xr[2 * S::SLOTS * ZB + 4 * slot + c.zw - 1];
            hxk = xr[o - 1];
        }
        if (lane == 31 && kb + 4 < ZP) epk = Ep[re + 4];
        float exb = 1.f, exa = 0.f, eyb = 1.f, eya = 0.f;
        if (XY) {
            exb = __ldg(xt + 2 * nx + i); exa = __ldg(xt + 3 * nx + i);
            eyb = __ldg(yt + 2 * ny + j); eya = __ldg(yt + 3 * ny + j);
        }
        {
            const float t0 = __shfl_up_sync(0xffffffffu, hy[3], 1);
            const float t1 = __shfl_up_sync(0xffffffffu, hx[3], 1);
            const float t2 = __shfl_down_sync(0xffffffffu, ep[0], 1);
            if (lane != 0) { hyk = t0; hxk = t1; }
            if (lane != 31) epk = t2;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = kb + q;
            const bool vzE = k < nz, vz = k <= nz - 2, kin = k >= 1 && k <= nz - 2;
            const float hym = (q == 0) ? hyk : hy[q - 1];
            const float hxkm = (q == 0) ? hxk : hx[q - 1];
            {
                float qy = 0.f, qz;
                const float dy = y3_d(hz[q], hzm[q], rdx);
                const float ty = XY ? y3_s(dy, eyb, eya, p6[q], qy) : dy;
                const float tz = y3_s(y3_d(hy[q], hym, rdx), ezb[q], eza[q], p7[q], qz);
                const bool v = xok && vzE;
                const float curl = y3_curl(ty, !jin, pmy, tz, !kin, pmz);
                const float en1 = y3_e(en[0][q], curl, dt, y3_ec(ep[q], epi[q]));
                en[0][q] = v ? en1 : en[0][q];
                if (XY) p6[q] = v ? qy : p6[q];
                p7[q] = v ? qz : p7[q];
            }
            {
                float qz, qx = 0.f;
                const float dx = y3_d(hz[q], c.hzp[q], rdx);
                const float tz = y3_s(y3_d(hx[q], hxkm, rdx), ezb[q], eza[q], p8[q], qz);
                const float tx = XY ? y3_s(dx, exb, exa, p9[q], qx) : dx;
                const bool v = vyH && vzE;
                const float curl = y3_curl(tz, !kin, pmz, tx, !iin, pmx);
                const float en1 = y3_e(en[1][q], curl, dt, y3_ec(ep[q], epj[q]));
                en[1][q] = v ? en1 : en[1][q];
                p8[q] = v ? qz : p8[q];
                if (XY) p9[q] = v ? qx : p9[q];
            }
            {
                float qx = 0.f, qy = 0.f;
                const float dx = y3_d(hy[q], c.hyp[q], rdx), dy = y3_d(hx[q], hxm[q], rdx);
                const float tx = XY ? y3_s(dx, exb, exa, p10[q], qx) : dx;
                const float ty = XY ? y3_s(dy, eyb, eya, p11[q], qy) : dy;
                const float curl = y3_curl(tx, !iin, pmx, ty, !jin, pmy);
                const float en1 = y3_e(en[2][q], curl, dt, y3_ec(ep[q], (q < 3) ? ep[q + 1] : epk));
                en[2][q] = vz ? en1 : en[2][q];
                if (XY) {
                    p10[q] = vz ? qx : p10[q];
                    p11[q] = vz ? qy : p11[q];
                }
            }
        }
        if (e0 < e1x) {
            const int cmp = P.src_comp;
            const float a = __ldg(amp);
            const float sgn = P.src_is_point ? (float)P.point_sign : -1.f;
            for (int e = e0; e < e1x; ++e) {
                const int kq = __ldg(P.src_col + e) - kb;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (kq != q) continue;
                    float epn;
                    if (cmp == 0) epn = epi[q];
                    else if (cmp == 1) epn = epj[q];
                    else epn = (q < 3) ? ep[q + 1] : epk;
                    const float ecomp = y3_ec(ep[q], epn);
                    const float v = __fmul_rn(a, __ldg(P.src_w + e));
#pragma unroll
                    for (int cc = 0; cc < 3; ++cc) {
                        if (cc != cmp) continue;
                        en[cc][q] = y3_src(en[cc][q], v, ecomp, P.src_is_point != 0, sgn);
                    }
                }
            }
        }
        if (act) {
            st4v(P.eo[0] + g, en[0]);
            st4v(P.eo[1] + g, en[1]);
            st4v(P.eo[2] + g, en[2]);
        }
        if (xok && bze) st4v(P.po[7] + g, p7);
        if (vyH && bze) st4v(P.po[8] + g, p8);
        if (XY) {
            if (xok && bye) st4v(P.po[6] + g, p6);
            if (vyH && bxe) st4v(P.po[9] + g, p9);
            if (bxe) st4v(P.po[10] + g, p10);
            if (bye) st4v(P.po[11] + g, p11);
        }
    }
    // H of this plane is the x-1 neighbour of the next one
#pragma unroll
    for (int q = 0; q < 4; ++q) { c.hyp[q] = hy[q]; c.hzp[q] = hz[q]; }
}

template <int V, int TY>
__global__ void __launch_bounds__(XmShape<V, TY>::THREADS, 1)
k_yee3d_xm(const __grid_constant__ Split3 P, const __grid_constant__ XmMaps M,
           const float *__restrict__ amp, int par, const int64_t *__restrict__ share,
           int *__restrict__ err) {
    using S = XmShape<V, TY>;
    extern __shared__ __align__(128) unsigned char xm_raw[];
    XmCtx c;
    c.stages = reinterpret_cast<float *>(xm_raw);
    c.xh = c.stages + XM_NS * S::STAGE;
    c.bars = reinterpret_cast<uint64_t *>(c.xh + 2 * S::XH);

    const int nx = P.nx, ny = P.ny, ZP = P.zp;
    const int64_t u0 = __ldg(share + blockIdx.x), u1 = __ldg(share + blockIdx.x + 1);
    if (u1 <= u0) return;
    XmSeq Q;
    Q.init(u0, u1, nx);

    c.tid = threadIdx.x;
    c.lane = c.tid & 31;
    const int w = c.tid >> 5;
    c.slot = w / V;
    c.zw = w % V;
    c.kb = c.zw * 128 + 4 * c.lane;
    // z-layer box of this lane's float4 (geometry, fixed per thread)
    c.pzo = c.kb < M.zl ? c.slot * XM_BZ + c.kb
                        : (c.kb >= M.zh ? S::PZB + c.slot * XM_BZ + (c.kb - M.zh) : 0);
    // masked z profiles of the own cells (H b, H a, E b, E a); (1, 0) past zpitch
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = c.kb + q;
            c.zp[a][q] = k < ZP ? __ldg(M.ptab + 4 * (nx + ny) + a * ZP + k) : ((a & 1) ? 0.f : 1.f);
        }

    // producer state (thread 0): next element to stage
    c.pt = Q.t0;
    c.pp = Q.first(c.pt);
    c.pmore = true;
    c.issued = 0;
    if (c.tid == 0) {
        for (int s = 0; s < XM_NS; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(xm_s32(c.bars + s)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (; c.issued < XM_NS - 1 && c.pmore; ++c.issued) {
            xm_issue<V, TY>(M, par, c.pt, c.pp, c.stages + c.issued * S::STAGE, c.bars + c.issued);
            c.pmore = Q.next(c.pt, c.pp);
        }
    }
    __syncthreads();

    c.ok = true;
    c.ready = 0;
    z4(c.hyp); z4(c.hzp);
    int t = Q.t0, p = Q.first(t);
    int xs = Q.xs(t), xe = Q.xe(t), last = Q.last(t);
    for (int n = 0;; ++n) {
        const bool halo = p < xs, tail = p >= xe;
        const bool has_next = p + 1 < nx && p + 1 <= last;
        if (p == xs - 1 || (xs == 0 && p == 0)) { z4(c.hyp); z4(c.hzp); }
        const int j = __ldg(M.ytab + t) - 1 + c.slot;
        const bool xy = inband(P.B, 0, 0, p) || inband(P.B, 0, 1, p) ||
                        (j >= 0 && j < ny && (inband(P.B, 1, 0, j) || inband(P.B, 1, 1, j)));
        if (xy)
            xm_elem<V, TY, true>(P, M, Q, c, n, t, p, halo, tail, has_next, amp, par, err);
        else
            xm_elem<V, TY, false>(P, M, Q, c, n, t, p, halo, tail, has_next, amp, par, err);
        const int tp = t;
        if (!Q.next(t, p)) break;
        if (t != tp) { xs = Q.xs(t); xe = Q.xe(t); last = Q.last(t); }
    }
    // copies still in flight after an expired wait: wait for them (bounded) before exit
    if (!c.ok && c.tid == 0) {
        const unsigned long long t0 = xm_clock();
        for (int m = max(c.issued - XM_NS, 0); m < c.issued; ++m)
            while (!xm_try(c.bars + m % XM_NS, (m / XM_NS) & 1) && xm_clock() - t0 < XM_WAIT_NS) {
            }
    }
}

}  // namespace mtb
