// Temporally blocked 2D Yee step (TM and TE) for sm_100a: up to TB_T time steps
// of the reference's step (TM core/stepper_tm.py:234-254, TE
// core/stepper_te.py:178-190, with CPML, soft sources and the monitor samples)
// per launch, each field value read from HBM once and written once per launch.
//
// Tiles. A tile is TB_R = 32 rows x TB_C = 128 columns of one structure's box
// arrays: its output block (TB_OUTR = 24 rows x TB_OUTC = 120 columns) with a
// TB_T-row halo above and below and a 4-column halo left and right. Every
// half step reads one neighbour on one side only, so after s sub-steps the
// cells at least s rows / columns inside the tile are still exact; the
// output block, TB_T rows and 4 columns in, is exact after TB_T sub-steps.
// Columns stay 4-aligned so every copy and every float4 access is 16-byte
// aligned.
//
// Block. One 1024-thread block per SM, persistent over a static share of the
// tiles: warp w owns tile row w, lane L columns 4L .. 4L+3. A thread keeps its
// cells' fields, 1/eps and x-layer CPML memory in registers for all sub-steps;
// the y-layer CPML memory (only lanes with a y-layer column touch it) stays in
// shared memory. Rows exchange through two shared-memory planes (TM: Ez for
// the row above's Hy update, Hy for the row below's Dz update; TE: Hz and Ey),
// two barriers per sub-step; columns exchange through warp shuffles.
//
// Staging. Everything a tile reads is brought into shared memory by the bulk
// copy engine, completion counted on one mbarrier: the field, 1/eps and CPML
// planes by TMA 2D tensor copies (cp.async.bulk.tensor.2d; rows and columns
// outside the array read as zero), and the structure's descriptor, its line
// samples and the tile's y profiles by 1D bulk copies (cp.async.bulk) from the
// plan's per-structure records. The next tile's copies are issued as soon as
// the current tile's planes have been moved to registers, so they overlap the
// current tile's sub-steps and stores; descriptors and profiles are double
// buffered for that. The y-layer CPML planes of a tile that reaches only one y
// layer are copied as a 32-column box. Waits are bounded by %globaltimer: an
// expired wait raises the plan's error flag, lets the copies in flight land
// (again bounded) and ends the block.
//
// Every launch reads buffer `par` of each ping-pong pair and writes buffer
// par ^ 1, whatever its sub-step count. Monitor samples of every sub-step go
// to consecutive ring slots, written by the thread owning the output cell.
#include <cuda.h>

namespace mtb {

constexpr int TB_T = 4;                      // sub-steps per launch (at most)
constexpr int TB_R = 32;                     // tile rows (one warp each)
constexpr int TB_C = 128;                    // tile columns (a float4 per lane)
constexpr int TB_OUTR = TB_R - 2 * TB_T;     // output rows per tile
constexpr int TB_OUTC = TB_C - 8;            // output columns per tile
constexpr int TB_NARROW = 32;                // columns of the narrow y-layer box
constexpr int TB_PLANE = TB_R * TB_C;        // floats per staged plane
constexpr int TB_THREADS = 32 * TB_R;
// tensor maps per structure: slot of each array (pairs are [buffer 0, buffer 1])
enum {
    TBM_MAIN = 0, TBM_X = 2, TBM_Y = 4, TBM_IEA = 6, TBM_IEB = 7,
    TBM_P1 = 8, TBM_P2 = 10, TBM_P0W = 12, TBM_P3W = 14, TBM_P0N = 16, TBM_P3N = 18,
    TBM_N = 20
};
// A tile is two int4: a = {structure, first output row r0, first output column
// c0, flags}; b = {bytes of the structure's record to copy, padded y-profile
// row length, float offset of the tile's y profiles (low, high 32 bits)}; the
// x-profile offset of the tile's first row follows in the tile's third int4:
// c = {offset low, high, padded x-profile row length, 0}.
constexpr int TB_WORK = 3;                   // int4 per tile
// work item flags (a.w)
constexpr int TBF_XPSI = 1;                  // x-layer CPML planes (psi 1, 2)
constexpr int TBF_YSHIFT = 1;                // bits 1-2: y-layer planes (psi 0, 3):
constexpr int TBF_YNONE = 0, TBF_YNARROW = 1, TBF_YWIDE = 2;   // none / narrow / full
constexpr int TBF_LEAN = 8;                  // bit 3: the whole tile is inside the grid's
                                             // updated cells and outside every CPML layer
constexpr int TBF_XS_SHIFT = 8;              // bits 8-15: narrow box start, columns past
                                             // the tile's first column
constexpr int TBF_LINE_SHIFT = 16;           // bits 16-31: line samples in the output block

// Per-structure record the kernels copy with one bulk copy: the descriptor and
// its line samples (the first n_lines used).
struct __align__(16) TbMeta {
    mtb_yee2d_struct s;
    mtb_line_sample lines[MAXL];
};
static_assert(sizeof(mtb_yee2d_struct) % 16 == 0, "descriptor copies are 16-byte multiples");
static_assert(sizeof(mtb_line_sample) % 16 == 0, "line copies are 16-byte multiples");

struct TbCtx {
    const TbMeta *meta;      // per structure
    const float *prof;       // padded profiles: per structure 4 y rows and 4 x rows
    const float *amp_e;      // coefficient row of sub-step 0; sub-step s at + s * ncols
    const float *amp_h;
    int ncols;
    int nsub;                // sub-steps this launch (1 .. TB_T)
    float *ring;             // ring slot of sub-step 0; sub-step s at + s * slot_elems
    int64_t slot_elems;
    int *err;
    int par;                 // buffer holding the old state
};

struct TbCtl {
    int4 rec[2][3];          // tile records, by tile parity (read ahead one tile)
    int4 cur[2];             // work item a of the tiles held in buffer sets 0, 1
    uint64_t bar;
    int ok;
};

template <bool TE>
constexpr int tb_nf() { return TE ? 5 : 4; }  // staged field planes incl. 1/eps
// shared memory: staged planes (fields, 1/eps, CPML psi 0..3), two row-exchange
// planes, the tile's y-layer CPML memory (psi 0, 3), two sets of y and x
// profiles and two records (double buffered), control
template <bool TE>
constexpr size_t tb_smem() {
    return sizeof(float) * ((size_t)TB_PLANE * (tb_nf<TE>() + 4 + 2 + 2) +
                            2 * 4 * (TB_C + TB_R)) +
           2 * sizeof(TbMeta) + sizeof(TbCtl);
}

__device__ __forceinline__ void tma2d(float *dst, const CUtensorMap *map, int x, int y,
                                      uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar)) : "memory");
}

// Shared-memory carve-up of the TB kernels.
template <bool TE>
struct TbLayout {
    float *stage, *xa, *xb, *yp, *prof, *xprof;
    TbMeta *meta;
    TbCtl *ctl;
    __device__ explicit TbLayout(unsigned char *raw) {
        stage = reinterpret_cast<float *>(raw);
        xa = stage + (tb_nf<TE>() + 4) * TB_PLANE;
        xb = xa + TB_PLANE;
        yp = xb + TB_PLANE;                      // psi 0 plane, psi 3 plane
        prof = yp + 2 * TB_PLANE;                // [2][hy b, hy a, ey b, ey a][TB_C]
        xprof = prof + 2 * 4 * TB_C;             // [2][hx b, hx a, ex b, ex a][TB_R]
        meta = reinterpret_cast<TbMeta *>(xprof + 2 * 4 * TB_R);  // [2]
        ctl = reinterpret_cast<TbCtl *>(meta + 2);
    }
};

// Issue tile (a, b, c)'s copies (one thread) into buffer set `bs` (record and
// profiles) and the staging planes; the same transaction brings the record of
// this block's following tile (`next`, if any) into rec[bs ^ 1].
template <bool TE>
__device__ __forceinline__ void tb_issue(const CUtensorMap *__restrict__ maps, const TbCtx &C,
                                         const int4 a, const int4 b, const int4 c,
                                         const int4 *__restrict__ work, int next, int n_work,
                                         TbLayout<TE> &L, int bs) {
    constexpr int NF = tb_nf<TE>();
    uint64_t *bar = &L.ctl->bar;
    const CUtensorMap *m = maps + (size_t)a.x * TBM_N;
    const int par = C.par;
    const int x0 = a.z - 4, y0 = a.y - TB_T;
    const int ymode = (a.w >> TBF_YSHIFT) & 3;
    const bool xl = a.w & TBF_XPSI;
    const uint32_t meta_bytes = (uint32_t)b.x;
    uint32_t bytes = NF * TB_PLANE * 4 + meta_bytes;
    if (xl) bytes += 2 * TB_PLANE * 4 + 4 * TB_R * 4;
    if (ymode == TBF_YWIDE) bytes += 2 * TB_PLANE * 4;
    if (ymode == TBF_YNARROW) bytes += 2 * TB_R * TB_NARROW * 4;
    if (ymode != TBF_YNONE) bytes += 4 * TB_C * 4;
    if (next < n_work) bytes += sizeof(int4) * TB_WORK;
    L.ctl->cur[bs] = a;
    mbar_expect_tx(bar, bytes);
    if (next < n_work)
        bulk_g2s(reinterpret_cast<float *>(L.ctl->rec[bs ^ 1]),
                 reinterpret_cast<const float *>(work + (size_t)TB_WORK * next),
                 sizeof(int4) * TB_WORK, bar);
    bulk_g2s(reinterpret_cast<float *>(L.meta + bs), reinterpret_cast<const float *>(C.meta + a.x),
             meta_bytes, bar);
    const CUtensorMap *fm[5] = {m + TBM_MAIN + par, m + TBM_X + par, m + TBM_Y + par,
                                m + TBM_IEA, m + TBM_IEB};
#pragma unroll
    for (int q = 0; q < NF; ++q) tma2d(L.stage + q * TB_PLANE, fm[q], x0, y0, bar);
    float *ps = L.stage + NF * TB_PLANE;     // CPML planes psi 0 .. 3
    if (xl) {
        tma2d(ps + 1 * TB_PLANE, m + TBM_P1 + par, x0, y0, bar);
        tma2d(ps + 2 * TB_PLANE, m + TBM_P2 + par, x0, y0, bar);
        // padded x profiles: row i of the structure sits at index i + 4
        const float *xp = C.prof + ((int64_t)(uint32_t)c.x | ((int64_t)c.y << 32));
        float *dst = L.xprof + bs * 4 * TB_R;
#pragma unroll
        for (int k = 0; k < 4; ++k) bulk_g2s(dst + k * TB_R, xp + (int64_t)k * c.z, TB_R * 4, bar);
    }
    if (ymode == TBF_YWIDE) {
        tma2d(ps, m + TBM_P0W + par, x0, y0, bar);
        tma2d(ps + 3 * TB_PLANE, m + TBM_P3W + par, x0, y0, bar);
    } else if (ymode == TBF_YNARROW) {
        const int xs = x0 + ((a.w >> TBF_XS_SHIFT) & 0xff);
        tma2d(ps, m + TBM_P0N + par, xs, y0, bar);
        tma2d(ps + 3 * TB_PLANE, m + TBM_P3N + par, xs, y0, bar);
    }
    if (ymode != TBF_YNONE) {
        // padded y profiles: column j of the structure sits at index j + 4
        const float *pp = C.prof + ((int64_t)(uint32_t)b.z | ((int64_t)b.w << 32));
        float *dst = L.prof + bs * 4 * TB_C;
#pragma unroll
        for (int k = 0; k < 4; ++k) bulk_g2s(dst + k * TB_C, pp + (int64_t)k * b.y, TB_C * 4, bar);
    }
}

// Thread 0 waits (bounded) for tile k's copies; block-uniform verdict in ctl->ok.
__device__ __forceinline__ void tb_wait(TbCtl &ctl, uint32_t parity, int *err) {
    bool ok = mbar_try_wait(&ctl.bar, parity);
    if (!ok) {
        const unsigned long long t0 = gtimer();
        while (!(ok = mbar_try_wait(&ctl.bar, parity)) && gtimer() - t0 < WAIT_NS) {
        }
        if (!ok) {
            atomicExch(err, 1);
            // let the copies in flight land before the block exits (bounded)
            const unsigned long long t1 = gtimer();
            while (!mbar_try_wait(&ctl.bar, parity) && gtimer() - t1 < WAIT_NS) {
            }
        }
    }
    ctl.ok = ok ? 1 : 0;
}

// Copy a staged float4 (plane a, this thread's cells) to registers.
__device__ __forceinline__ void tb_take(const float *stage, int a, int cell, float (&v)[4]) {
    lds4(stage + a * TB_PLANE + cell, v);
}

// CPML memory of this thread's cells: psi 1, 2 (x layers) to registers; psi 0, 3
// (y layers) to the tile's work planes yp (zero where not staged).
__device__ __forceinline__ void tb_take_psi(const float *ps, int flags, int w, int lane,
                                            float (&p1)[4], float (&p2)[4], float *yp) {
    const int cell = w * TB_C + 4 * lane;
    zero4(p1); zero4(p2);
    if (flags & TBF_XPSI) {
        tb_take(ps, 1, cell, p1);
        tb_take(ps, 2, cell, p2);
    }
    float p0[4], p3[4];
    zero4(p0); zero4(p3);
    const int ymode = (flags >> TBF_YSHIFT) & 3;
    if (ymode == TBF_YWIDE) {
        tb_take(ps, 0, cell, p0);
        tb_take(ps, 3, cell, p3);
    } else if (ymode == TBF_YNARROW) {
        const int rel = 4 * lane - ((flags >> TBF_XS_SHIFT) & 0xff);
        if (rel >= 0 && rel < TB_NARROW) {
            lds4(ps + w * TB_NARROW + rel, p0);
            lds4(ps + 3 * TB_PLANE + w * TB_NARROW + rel, p3);
        }
    }
    if (ymode != TBF_YNONE) {
        st4(yp + cell, p0);
        st4(yp + TB_PLANE + cell, p3);
    }
}

// Copy this row's values of component `comp` into the line samples of `mask`.
__device__ __forceinline__ void tb_sample(const mtb_line_sample *L, unsigned mask, int comp,
                                          int i, int jb, const float (&v)[4], float *ring) {
    while (mask) {
        const int l = __ffs(mask) - 1;
        mask &= mask - 1;
        const mtb_line_sample &s = L[l];
        if (s.comp != comp) continue;
        if (s.kind == 0) {
            if (s.index != i) continue;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j = jb + q;
                if (j >= s.lo && j < s.hi) ring[s.ring_off + (j - s.lo)] = v[q];
            }
        } else {
            if (i < s.lo || i >= s.hi) continue;
            const int q = s.index - jb;
#pragma unroll
            for (int qq = 0; qq < 4; ++qq)
                if (q == qq) ring[s.ring_off + (i - s.lo)] = v[qq];
        }
    }
}

// Tile start, common to TM and TE: thread 0's bounded wait for tile k's copies,
// the block-uniform verdict, and each thread's acquire of the completed phase.
template <bool TE>
__device__ __forceinline__ bool tb_begin(uint32_t k, TbLayout<TE> &L, int *err) {
    if (threadIdx.x == 0) tb_wait(*L.ctl, k & 1, err);
    __syncthreads();
    if (!L.ctl->ok) return false;
    (void)mbar_try_wait(&L.ctl->bar, k & 1);     // completed: acquire for this thread
    return true;
}

// Block start, common to TM and TE: barrier init and the first tile's copies
// (with the second tile's record).
template <bool TE>
__device__ __forceinline__ void tb_start(const CUtensorMap *__restrict__ maps, const TbCtx &C,
                                         const int4 *__restrict__ work, int n_work,
                                         TbLayout<TE> &L) {
    if (threadIdx.x == 0) {
        mbar_init(&L.ctl->bar, 1);
        mbar_fence_init();
        const int4 *r = work + (size_t)TB_WORK * blockIdx.x;
        tb_issue<TE>(maps, C, __ldg(r), __ldg(r + 1), __ldg(r + 2), work,
                     blockIdx.x + gridDim.x, n_work, L, 0);
    }
}

// After tile k's planes are taken: thread 0 issues tile k+1's copies from its
// record, which arrived with tile k's.
template <bool TE>
__device__ __forceinline__ void tb_next(const CUtensorMap *__restrict__ maps, const TbCtx &C,
                                        const int4 *__restrict__ work, int n_work, int it,
                                        uint32_t k, TbLayout<TE> &L) {
    if (threadIdx.x != 0 || it + (int)gridDim.x >= n_work) return;
    const int bs = (k + 1) & 1;
    const int4 *r = L.ctl->rec[bs];
    tb_issue<TE>(maps, C, r[0], r[1], r[2], work, it + 2 * gridDim.x, n_work, L, bs);
}

// ------------------------------------------------------------------ TM
// Per sub-step (reference order): Hx, Hy(n+1/2) from Ez(n) (core/stepper_tm.py:
// 85-128) with the magnetic sheet sources; Dz(n+1) from H(n+1/2) with PEC walls
// (:130-166); the electric source (:197-200); Ez = Dz / eps (:224-231).
__global__ void __launch_bounds__(TB_THREADS, 1) k_tb_tm(
    const CUtensorMap *__restrict__ maps, const int4 *__restrict__ work, int n_work, TbCtx C) {
    extern __shared__ __align__(1024) unsigned char tb_raw[];
    constexpr int NF = tb_nf<false>();
    TbLayout<false> L(tb_raw);
    float *xe = L.xa, *xh = L.xb;                     // Ez rows, Hy rows
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    int it = blockIdx.x;
    if (it >= n_work) return;
    tb_start<false>(maps, C, work, n_work, L);
    const int par = C.par, pn = par ^ 1;
    const int cell = w * TB_C + 4 * lane;             // this thread's offset in a plane
    for (uint32_t k = 0; it < n_work; ++k, it += gridDim.x) {
        if (!tb_begin<false>(k, L, C.err)) return;
        const int4 wk = L.ctl->cur[k & 1];
        const TbMeta &M = L.meta[k & 1];
        const mtb_yee2d_struct &S = M.s;
        float dz[4], hx[4], hy[4], ie[4], p1[4], p2[4];
        tb_take(L.stage, 0, cell, dz);
        tb_take(L.stage, 1, cell, hx);
        tb_take(L.stage, 2, cell, hy);
        tb_take(L.stage, 3, cell, ie);
        tb_take_psi(L.stage + NF * TB_PLANE, wk.w, w, lane, p1, p2, L.yp);
        __syncthreads();                                // staging planes are free
        tb_next<false>(maps, C, work, n_work, it, k, L);

        const int nx = S.nx, ny = S.ny, P = S.pitch;
        const int i = wk.y - TB_T + w;
        const int jb = wk.z - 4 + 4 * lane;
        const bool act = jb >= 0 && jb < P;
        const bool rowIn = i >= 0 && i < nx;
        const bool hyRow = i >= 0 && i <= nx - 2, dzRow = i >= 1 && i <= nx - 2;
        const float dt = S.dt, rdx = 1.0f / S.dx;
        unsigned mHx = 0, mHy = 0, mD = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = jb + q;
            if (rowIn && j >= 0 && j <= ny - 2) mHx |= 1u << q;
            if (hyRow && j >= 0 && j < ny) mHy |= 1u << q;
            if (dzRow && j >= 1 && j <= ny - 2) mD |= 1u << q;
        }
        // x profiles (warp-uniform: one row per warp)
        const bool bxH = hyRow && in_band(i, S.xband[0], S.xband[1]);
        const bool bxE = dzRow && in_band(i, S.xband[2], S.xband[3]);
        const float *xpr = L.xprof + (k & 1) * 4 * TB_R + w;
        const float hxb = bxH ? xpr[0] : 1.f, hxa = bxH ? xpr[TB_R] : 0.f;
        const float exb = bxE ? xpr[2 * TB_R] : 1.f, exa = bxE ? xpr[3 * TB_R] : 0.f;
        const bool byH = act && band4(jb, S.yband[0], S.yband[1]);
        const bool byE = act && dzRow && band4(jb, S.yband[2], S.yband[3]);
        // every lane of a tile that reaches a y layer runs the CPML arithmetic (inert
        // profiles and zero memory off the layer give the plain update): no divergence
        const bool yl = ((wk.w >> TBF_YSHIFT) & 3) != TBF_YNONE;
        float *yp0 = L.yp + cell, *yp3 = L.yp + TB_PLANE + cell;
        const float *pr = L.prof + (k & 1) * 4 * TB_C + 4 * lane;
        const bool outC = act && lane >= 1 && lane <= 30;
        const bool out = outC && rowIn && w >= TB_T && w < TB_T + TB_OUTR;
        const unsigned lmask = (unsigned)wk.w >> TBF_LINE_SHIFT;
        const uint32_t ro = (uint32_t)(i * P + jb);
        const bool srcE = act && rowIn && S.src_e.n > 0 && i >= S.src_e.row_lo &&
                          i <= S.src_e.row_hi;
        const bool srcH1 = act && hyRow && S.src_h1.n > 0 && i >= S.src_h1.row_lo &&
                           i <= S.src_h1.row_hi;
        const bool srcH2 = act && rowIn && S.src_h2.n > 0 && i >= S.src_h2.row_lo &&
                           i <= S.src_h2.row_hi;
        if (wk.w & TBF_LEAN) {
            // every cell of the tile is updated and no CPML term is active: the
            // same arithmetic without validity masks or CPML memory
            float *rs0 = (out && S.ring_full[0] >= 0) ? C.ring + S.ring_full[0] + ro : nullptr;
            float *rs1 = (out && S.ring_full[1] >= 0) ? C.ring + S.ring_full[1] + ro : nullptr;
            float *rs2 = (out && S.ring_full[2] >= 0) ? C.ring + S.ring_full[2] + ro : nullptr;
            for (int s = 0; s < C.nsub; ++s) {
                float ez[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) ez[q] = dz[q] * ie[q];
                st4(xe + cell, ez);
                __syncthreads();
                float eb[4];
                if (w + 1 < TB_R) lds4(xe + cell + TB_C, eb);
                else zero4(eb);
                const float ezR = __shfl_down_sync(0xffffffffu, ez[0], 1);
                const float *ah = C.amp_h + s * C.ncols;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float er = (q < 3) ? ez[q + 1] : ezR;
                    hx[q] = hx[q] - dt * ((er - ez[q]) * rdx);
                    hy[q] = hy[q] + dt * ((eb[q] - ez[q]) * rdx);
                }
                if (srcH2) apply_cells(S.src_h2, i, ah, jb, hx);
                if (srcH1) apply_cells(S.src_h1, i, ah, jb, hy);
                st4(xh + cell, hy);
                __syncthreads();
                float ha[4];
                if (w > 0) lds4(xh + cell - TB_C, ha);
                else zero4(ha);
                const float hxm0 = __shfl_up_sync(0xffffffffu, hx[3], 1);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float hxm = (q == 0) ? hxm0 : hx[q - 1];
                    const float dhy = (hy[q] - ha[q]) * rdx;
                    const float dhx = (hx[q] - hxm) * rdx;
                    dz[q] = dz[q] + dt * (dhy - dhx);
                }
                if (srcE) apply_cells(S.src_e, i, C.amp_e + s * C.ncols, jb, dz);
                if (out) {
                    float ezN[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) ezN[q] = dz[q] * ie[q];
                    const int64_t so = s * C.slot_elems;
                    if (rs0) st4(rs0 + so, ezN);
                    if (rs1) st4(rs1 + so, hx);
                    if (rs2) st4(rs2 + so, hy);
                    if (lmask) {
                        float *ring = C.ring + so;
                        tb_sample(M.lines, lmask, MTB_C2_MAIN, i, jb, ezN, ring);
                        tb_sample(M.lines, lmask, MTB_C2_X, i, jb, hx, ring);
                        tb_sample(M.lines, lmask, MTB_C2_Y, i, jb, hy, ring);
                    }
                }
            }
        } else
        for (int s = 0; s < C.nsub; ++s) {
            float ez[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) ez[q] = dz[q] * ie[q];
            st4(xe + cell, ez);
            __syncthreads();
            float eb[4];
            if (w + 1 < TB_R) lds4(xe + cell + TB_C, eb);
            else zero4(eb);
            const float ezR = __shfl_down_sync(0xffffffffu, ez[0], 1);   // lane 31: halo
            const float *ah = C.amp_h + s * C.ncols;
            // Hx(n+1/2)
            if (yl) {
                float p0[4], b[4], a[4];
                lds4(yp0, p0);
                lds4(pr, b);
                lds4(pr + TB_C, a);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float er = (q < 3) ? ez[q + 1] : ezR;
                    const float d = (er - ez[q]) * rdx;
                    const float pv = b[q] * p0[q] + a[q] * d;
                    const float hn = hx[q] - dt * (d + pv);
                    const bool v = (mHx >> q) & 1u;
                    hx[q] = v ? hn : hx[q];
                    p0[q] = v ? pv : p0[q];
                }
                st4(yp0, p0);
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float er = (q < 3) ? ez[q + 1] : ezR;
                    const float hn = hx[q] - dt * ((er - ez[q]) * rdx);
                    hx[q] = ((mHx >> q) & 1u) ? hn : hx[q];
                }
            }
            if (srcH2) apply_cells(S.src_h2, i, ah, jb, hx);
            // Hy(n+1/2)
            if (bxH) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float d = (eb[q] - ez[q]) * rdx;
                    const float pv = hxb * p1[q] + hxa * d;
                    const float hn = hy[q] + dt * (d + pv);
                    const bool v = (mHy >> q) & 1u;
                    hy[q] = v ? hn : hy[q];
                    p1[q] = v ? pv : p1[q];
                }
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float hn = hy[q] + dt * ((eb[q] - ez[q]) * rdx);
                    hy[q] = ((mHy >> q) & 1u) ? hn : hy[q];
                }
            }
            if (srcH1) apply_cells(S.src_h1, i, ah, jb, hy);
            st4(xh + cell, hy);
            __syncthreads();
            float ha[4];
            if (w > 0) lds4(xh + cell - TB_C, ha);
            else zero4(ha);
            const float hxm0 = __shfl_up_sync(0xffffffffu, hx[3], 1);     // lane 0: halo
            // Dz(n+1)
            if (yl || bxE) {
                float p3[4], b3[4], a3[4];
                if (yl) {
                    lds4(yp3, p3);
                    lds4(pr + 2 * TB_C, b3);
                    lds4(pr + 3 * TB_C, a3);
                } else {
                    zero4(p3); zero4(a3);
                    b3[0] = b3[1] = b3[2] = b3[3] = 1.f;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float hxm = (q == 0) ? hxm0 : hx[q - 1];
                    const float dhy = (hy[q] - ha[q]) * rdx;
                    const float dhx = (hx[q] - hxm) * rdx;
                    const float q2 = exb * p2[q] + exa * dhy;
                    const float q3 = b3[q] * p3[q] + a3[q] * dhx;
                    const float curl = (dhy + q2) - (dhx + q3);
                    const float dn = dz[q] + dt * curl;
                    const bool v = (mD >> q) & 1u;
                    dz[q] = v ? dn : dz[q];
                    p2[q] = v ? q2 : p2[q];
                    p3[q] = v ? q3 : p3[q];
                }
                if (yl) st4(yp3, p3);
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float hxm = (q == 0) ? hxm0 : hx[q - 1];
                    const float dhy = (hy[q] - ha[q]) * rdx;
                    const float dhx = (hx[q] - hxm) * rdx;
                    const float dn = dz[q] + dt * (dhy - dhx);
                    dz[q] = ((mD >> q) & 1u) ? dn : dz[q];
                }
            }
            if (srcE) apply_cells(S.src_e, i, C.amp_e + s * C.ncols, jb, dz);
            if (out) {
                float ezN[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) ezN[q] = dz[q] * ie[q];
                float *ring = C.ring + s * C.slot_elems;
                if (S.ring_full[0] >= 0) st4(ring + S.ring_full[0] + ro, ezN);
                if (S.ring_full[1] >= 0) st4(ring + S.ring_full[1] + ro, hx);
                if (S.ring_full[2] >= 0) st4(ring + S.ring_full[2] + ro, hy);
                if (lmask) {
                    tb_sample(M.lines, lmask, MTB_C2_MAIN, i, jb, ezN, ring);
                    tb_sample(M.lines, lmask, MTB_C2_X, i, jb, hx, ring);
                    tb_sample(M.lines, lmask, MTB_C2_Y, i, jb, hy, ring);
                }
            }
        }
        if (out) {
            st4(S.f_main[pn] + ro, dz);
            st4(S.f_x[pn] + ro, hx);
            st4(S.f_y[pn] + ro, hy);
            float t[4];
            if (byH) { lds4(yp0, t); st4(S.psi[0][pn] + ro, t); }
            if (bxH) st4(S.psi[1][pn] + ro, p1);
            if (bxE) st4(S.psi[2][pn] + ro, p2);
            if (byE) { lds4(yp3, t); st4(S.psi[3][pn] + ro, t); }
        }
        __syncthreads();                                // records, exchange planes reused
    }
}

// ------------------------------------------------------------------ TE
// Per sub-step (reference order, core/stepper_te.py:178-190): Dx, Dy(n+1/2)
// from Hz(n) with CPML (:73-111), the source into Dy (:120-134), E = D / eps
// (:150-175); Hz(n+1) from E(n+1/2) (:113-117) with the magnetic sheet source.
__global__ void __launch_bounds__(TB_THREADS, 1) k_tb_te(
    const CUtensorMap *__restrict__ maps, const int4 *__restrict__ work, int n_work, TbCtx C) {
    extern __shared__ __align__(1024) unsigned char tb_raw[];
    constexpr int NF = tb_nf<true>();
    TbLayout<true> L(tb_raw);
    float *xz = L.xa, *xy = L.xb;                     // Hz rows, Ey rows
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    int it = blockIdx.x;
    if (it >= n_work) return;
    tb_start<true>(maps, C, work, n_work, L);
    const int par = C.par, pn = par ^ 1;
    const int cell = w * TB_C + 4 * lane;
    for (uint32_t k = 0; it < n_work; ++k, it += gridDim.x) {
        if (!tb_begin<true>(k, L, C.err)) return;
        const int4 wk = L.ctl->cur[k & 1];
        const TbMeta &M = L.meta[k & 1];
        const mtb_yee2d_struct &S = M.s;
        float hz[4], dx[4], dy[4], ix[4], iy[4], p1[4], p2[4];
        tb_take(L.stage, 0, cell, hz);
        tb_take(L.stage, 1, cell, dx);
        tb_take(L.stage, 2, cell, dy);
        tb_take(L.stage, 3, cell, ix);
        tb_take(L.stage, 4, cell, iy);
        tb_take_psi(L.stage + NF * TB_PLANE, wk.w, w, lane, p1, p2, L.yp);
        __syncthreads();
        tb_next<true>(maps, C, work, n_work, it, k, L);

        const int nx = S.nx, ny = S.ny, P = S.pitch;
        const int i = wk.y - TB_T + w;
        const int jb = wk.z - 4 + 4 * lane;
        const bool act = jb >= 0 && jb < P;
        const bool rowIn = i >= 0 && i < nx;
        const bool hzRow = i >= 0 && i <= nx - 2, dyRow = i >= 1 && i <= nx - 2;
        const float dt = S.dt, rdx = 1.0f / S.dx;
        unsigned mX = 0, mY = 0, mZ = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = jb + q;
            if (hzRow && j >= 1 && j <= ny - 2) mX |= 1u << q;
            if (dyRow && j >= 0 && j <= ny - 2) mY |= 1u << q;
            if (hzRow && j >= 0 && j <= ny - 2) mZ |= 1u << q;
        }
        const bool bxH = hzRow && in_band(i, S.xband[0], S.xband[1]);
        const bool bxE = dyRow && in_band(i, S.xband[2], S.xband[3]);
        const float *xpr = L.xprof + (k & 1) * 4 * TB_R + w;
        const float hxb = bxH ? xpr[0] : 1.f, hxa = bxH ? xpr[TB_R] : 0.f;
        const float exb = bxE ? xpr[2 * TB_R] : 1.f, exa = bxE ? xpr[3 * TB_R] : 0.f;
        const bool byE = act && hzRow && band4(jb, S.yband[2], S.yband[3]);
        const bool byH = act && hzRow && band4(jb, S.yband[0], S.yband[1]);
        // every lane of a tile that reaches a y layer runs the CPML arithmetic (inert
        // profiles and zero memory off the layer give the plain update): no divergence
        const bool yl = ((wk.w >> TBF_YSHIFT) & 3) != TBF_YNONE;
        float *yp0 = L.yp + cell, *yp3 = L.yp + TB_PLANE + cell;
        const float *pr = L.prof + (k & 1) * 4 * TB_C + 4 * lane;
        const bool outC = act && lane >= 1 && lane <= 30;
        const bool out = outC && rowIn && w >= TB_T && w < TB_T + TB_OUTR;
        const unsigned lmask = (unsigned)wk.w >> TBF_LINE_SHIFT;
        const uint32_t ro = (uint32_t)(i * P + jb);
        const bool srcE = act && rowIn && S.src_e.n > 0 && i >= S.src_e.row_lo &&
                          i <= S.src_e.row_hi;
        const bool srcH = act && hzRow && S.src_h1.n > 0 && i >= S.src_h1.row_lo &&
                          i <= S.src_h1.row_hi;
        if (wk.w & TBF_LEAN) {
            // every cell of the tile is updated and no CPML term is active
            float *rs0 = (out && S.ring_full[0] >= 0) ? C.ring + S.ring_full[0] + ro : nullptr;
            float *rs1 = (out && S.ring_full[1] >= 0) ? C.ring + S.ring_full[1] + ro : nullptr;
            float *rs2 = (out && S.ring_full[2] >= 0) ? C.ring + S.ring_full[2] + ro : nullptr;
            for (int s = 0; s < C.nsub; ++s) {
                st4(xz + cell, hz);
                __syncthreads();
                float ha[4];
                if (w > 0) lds4(xz + cell - TB_C, ha);
                else zero4(ha);
                const float hzL = __shfl_up_sync(0xffffffffu, hz[3], 1);
                float ex[4], ey[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float hm = (q == 0) ? hzL : hz[q - 1];
                    dx[q] = dx[q] + dt * ((hz[q] - hm) * rdx);
                    ex[q] = dx[q] * ix[q];
                    dy[q] = dy[q] - dt * ((hz[q] - ha[q]) * rdx);
                }
                if (srcE) apply_cells(S.src_e, i, C.amp_e + s * C.ncols, jb, dy);
#pragma unroll
                for (int q = 0; q < 4; ++q) ey[q] = dy[q] * iy[q];
                st4(xy + cell, ey);
                __syncthreads();
                float eb[4];
                if (w + 1 < TB_R) lds4(xy + cell + TB_C, eb);
                else zero4(eb);
                const float exR = __shfl_down_sync(0xffffffffu, ex[0], 1);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float exn = (q < 3) ? ex[q + 1] : exR;
                    const float dey = (eb[q] - ey[q]) * rdx;
                    const float dex = (exn - ex[q]) * rdx;
                    hz[q] = hz[q] - dt * (dey - dex);
                }
                if (srcH) apply_cells(S.src_h1, i, C.amp_h + s * C.ncols, jb, hz);
                if (out) {
                    const int64_t so = s * C.slot_elems;
                    if (rs0) st4(rs0 + so, hz);
                    if (rs1) st4(rs1 + so, ex);
                    if (rs2) st4(rs2 + so, ey);
                    if (lmask) {
                        float *ring = C.ring + so;
                        tb_sample(M.lines, lmask, MTB_C2_MAIN, i, jb, hz, ring);
                        tb_sample(M.lines, lmask, MTB_C2_X, i, jb, ex, ring);
                        tb_sample(M.lines, lmask, MTB_C2_Y, i, jb, ey, ring);
                    }
                }
            }
        } else
        for (int s = 0; s < C.nsub; ++s) {
            st4(xz + cell, hz);
            __syncthreads();
            float ha[4];
            if (w > 0) lds4(xz + cell - TB_C, ha);
            else zero4(ha);
            const float hzL = __shfl_up_sync(0xffffffffu, hz[3], 1);       // lane 0: halo
            // Dx / Ex(n+1/2)
            if (yl) {
                float p0[4], b[4], a[4];
                lds4(yp0, p0);
                lds4(pr + 2 * TB_C, b);
                lds4(pr + 3 * TB_C, a);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float hm = (q == 0) ? hzL : hz[q - 1];
                    const float d = (hz[q] - hm) * rdx;
                    const float pv = b[q] * p0[q] + a[q] * d;
                    const float dn = dx[q] + dt * (d + pv);
                    const bool v = (mX >> q) & 1u;
                    dx[q] = v ? dn : dx[q];
                    p0[q] = v ? pv : p0[q];
                }
                st4(yp0, p0);
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float hm = (q == 0) ? hzL : hz[q - 1];
                    const float dn = dx[q] + dt * ((hz[q] - hm) * rdx);
                    dx[q] = ((mX >> q) & 1u) ? dn : dx[q];
                }
            }
            float ex[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) ex[q] = hzRow ? dx[q] * ix[q] : 0.f;
            // Dy / Ey(n+1/2), source into Dy
            if (bxE) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float d = (hz[q] - ha[q]) * rdx;
                    const float pv = exb * p1[q] + exa * d;
                    const float dn = dy[q] - dt * (d + pv);
                    const bool v = (mY >> q) & 1u;
                    dy[q] = v ? dn : dy[q];
                    p1[q] = v ? pv : p1[q];
                }
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float dn = dy[q] - dt * ((hz[q] - ha[q]) * rdx);
                    dy[q] = ((mY >> q) & 1u) ? dn : dy[q];
                }
            }
            if (srcE) apply_cells(S.src_e, i, C.amp_e + s * C.ncols, jb, dy);
            float ey[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) ey[q] = rowIn ? dy[q] * iy[q] : 0.f;
            st4(xy + cell, ey);
            __syncthreads();
            float eb[4];
            if (w + 1 < TB_R) lds4(xy + cell + TB_C, eb);
            else zero4(eb);
            const float exR = __shfl_down_sync(0xffffffffu, ex[0], 1);     // lane 31: halo
            // Hz(n+1)
            if (yl || bxH) {
                float p3[4], b3[4], a3[4];
                if (yl) {
                    lds4(yp3, p3);
                    lds4(pr, b3);
                    lds4(pr + TB_C, a3);
                } else {
                    zero4(p3); zero4(a3);
                    b3[0] = b3[1] = b3[2] = b3[3] = 1.f;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float exn = (q < 3) ? ex[q + 1] : exR;
                    const float dey = (eb[q] - ey[q]) * rdx;
                    const float dex = (exn - ex[q]) * rdx;
                    const float q2 = hxb * p2[q] + hxa * dey;
                    const float q3 = b3[q] * p3[q] + a3[q] * dex;
                    const float cz = (dey + q2) - (dex + q3);
                    const float hn = hz[q] - dt * cz;
                    const bool v = (mZ >> q) & 1u;
                    hz[q] = v ? hn : hz[q];
                    p2[q] = v ? q2 : p2[q];
                    p3[q] = v ? q3 : p3[q];
                }
                if (yl) st4(yp3, p3);
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float exn = (q < 3) ? ex[q + 1] : exR;
                    const float dey = (eb[q] - ey[q]) * rdx;
                    const float dex = (exn - ex[q]) * rdx;
                    const float hn = hz[q] - dt * (dey - dex);
                    hz[q] = ((mZ >> q) & 1u) ? hn : hz[q];
                }
            }
            if (srcH) apply_cells(S.src_h1, i, C.amp_h + s * C.ncols, jb, hz);
            if (out) {
                float *ring = C.ring + s * C.slot_elems;
                if (S.ring_full[0] >= 0) st4(ring + S.ring_full[0] + ro, hz);
                if (S.ring_full[1] >= 0) st4(ring + S.ring_full[1] + ro, ex);
                if (S.ring_full[2] >= 0) st4(ring + S.ring_full[2] + ro, ey);
                if (lmask) {
                    tb_sample(M.lines, lmask, MTB_C2_MAIN, i, jb, hz, ring);
                    tb_sample(M.lines, lmask, MTB_C2_X, i, jb, ex, ring);
                    tb_sample(M.lines, lmask, MTB_C2_Y, i, jb, ey, ring);
                }
            }
        }
        if (out) {
            st4(S.f_main[pn] + ro, hz);
            st4(S.f_x[pn] + ro, dx);
            st4(S.f_y[pn] + ro, dy);
            float t[4];
            if (byE) { lds4(yp0, t); st4(S.psi[0][pn] + ro, t); }
            if (bxE) st4(S.psi[1][pn] + ro, p1);
            if (bxH) st4(S.psi[2][pn] + ro, p2);
            if (byH) { lds4(yp3, t); st4(S.psi[3][pn] + ro, t); }
        }
        __syncthreads();
    }
}

}  // namespace mtb
