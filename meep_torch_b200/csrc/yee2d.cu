// Batched 2D Yee step (TM and TE) for sm_100a.
//
// One warp marches down rows i0..i1-1 of a 128-column strip of one
// structure: lane L owns columns c0+4L .. c0+4L+3. Each iteration fuses the
// reference's whole step for one row:
//   TM (core/stepper_tm.py:234-254): H(n+1/2) of row i from Ez(n) of rows
//      i, i+1 -> magnetic sheet source -> Dz(n+1) of row i from H rows
//      i-1, i -> electric source -> Ez = Dz / eps.
//   TE (core/stepper_te.py:178-190): D/E(n+1/2) of row i+1 from Hz(n) rows
//      i, i+1 -> source into Dy -> E = D / eps -> Hz(n+1) of row i.
// Ez (TM) and Ex/Ey (TE) are not stored: they are D * (1/eps), recomputed
// where needed, so the per-cell traffic is read+write of the three stored
// fields plus one (TM) or two (TE) 1/eps reads.
//
// Input rows are staged in shared memory by a per-warp pipeline of bulk
// copies (cp.async.bulk, completion counted on one mbarrier per stage):
// NST stages, each holding one row of every input array over the column
// window c0-4 .. c0+131 (the strip plus the 4-aligned halo the stencil needs),
// issued NST-1 rows ahead of use. Waits are bounded by %globaltimer; a wait
// that expires raises the plan's error flag and the warp stops.
// Halo values (the row above the strip, the columns left/right of it) are
// recomputed from the neighbours' old values, which is why every evolving
// array is a ping-pong pair. CPML memory is only touched where its profile is
// active (a != 0 or b != 1); outside the layers it is identically zero, as in
// the reference.
#include <algorithm>
#include <cstring>
#include <mutex>

#include <cudaTypedefs.h>
#include <vector>

#include "mtb_common.cuh"

namespace mtb {

constexpr int MAXL = 16;          // line samples per structure
constexpr int WARPS2D = 4;        // warps per block
constexpr int NST = 4;            // pipeline stages per warp
constexpr int EXT = 136;          // staged row: columns c0-4 .. c0+131
constexpr unsigned long long WAIT_NS = 2000000000ull;   // bounded wait: 2 s

struct Ctx2D {
    const float *amp_e;           // coefficient row of this step [n_cols]
    const float *amp_h;
    float *ring;                  // ring slot of this step
    int *err;                     // device error flag (1 = a bounded wait expired)
    int par;                      // buffer holding the old state
    int first;                    // first step executed by the plan
    int wr;                       // tile kernels: rows per warp (1 or WROWS)
    int pst;                      // pole buffer holding P(n) (0..2)
};

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(float *dst, const float *src, uint32_t bytes,
                                         uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void ld4(const float *p, float (&v)[4]) {
    const float4 x = *reinterpret_cast<const float4 *>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void lds4(const float *p, float (&v)[4]) {   // shared memory
    const float4 x = *reinterpret_cast<const float4 *>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void st4(float *p, const float (&v)[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void zero4(float (&v)[4]) { v[0] = v[1] = v[2] = v[3] = 0.f; }
__device__ __forceinline__ void copy4(float (&d)[4], const float (&s)[4]) {
    d[0] = s[0]; d[1] = s[1]; d[2] = s[2]; d[3] = s[3];
}

// ---------------------------------------------------------------- row pipeline
// Rows r = i0-1+k (k = 0 .. nrows-1) go through stage k % NST. Rows outside
// [0, nx) get an arrive without a copy so every stage's phase parity stays
// k / NST; their shared data is never read.
template <int NA>
struct Pipe {
    float *buf;                   // NST * NA * EXT floats (this warp's)
    uint64_t *bar;                // NST mbarriers
    const float *const *src;      // base of each staged global array (shared memory)
    int64_t P;                    // row pitch
    int w0;                       // first staged global column
    int dst;                      // float offset of w0 inside a staged row
    uint32_t bytes;               // bytes per staged row copy
    int i0m1, nx, nrows;
    int lane;
    static constexpr int STG = NA * EXT;

    // lane 0 arms the stage's barrier, lanes 0..NA-1 each issue one array's copy
    __device__ void issue(int k) const {
        if (k >= nrows) return;
        const int r = i0m1 + k;
        uint64_t *b = bar + (k % NST);
        if (r < 0 || r >= nx) {
            if (lane == 0) mbar_arrive(b);
            return;
        }
        if (lane == 0) mbar_expect_tx(b, bytes * NA);
        if (lane < NA)
            bulk_g2s(buf + (k % NST) * STG + lane * EXT + dst, src[lane] + r * P + w0, bytes, b);
    }
    // true when stage k is ready; false (error flag raised) when the bounded
    // wait expired
    __device__ bool wait(int k, int *err) const {
        uint64_t *b = bar + (k % NST);
        const uint32_t par = (k / NST) & 1;
        if (mbar_try_wait(b, par)) return true;
        const unsigned long long t0 = gtimer();
        while (!mbar_try_wait(b, par)) {
            if (gtimer() - t0 > WAIT_NS) {
                if (lane == 0) atomicExch(err, 1);
                return false;
            }
        }
        return true;
    }
    // after an expired wait: let this warp's copies in flight land (bounded)
    __device__ void drain(int k_from, int k_to) const {
        for (int k = k_from; k < k_to && k < nrows; ++k) {
            uint64_t *b = bar + (k % NST);
            const uint32_t par = (k / NST) & 1;
            const unsigned long long t0 = gtimer();
            while (!mbar_try_wait(b, par) && gtimer() - t0 < WAIT_NS) {
            }
        }
    }
    __device__ const float *row(int k, int a) const { return buf + (k % NST) * STG + a * EXT; }
};

// F[row, jb+q] -= amp * w for the cells of `row` in `cl` (CSR by row).
// First e in [e0, e1) whose column is >= key (the columns of a row ascend: the
// plan rejects other orders); e1 if there is none. Every probe stays in [e0, e1).
__device__ __forceinline__ int lower_col(const int32_t *__restrict__ col, int e0, int e1,
                                         int key) {
    while (e0 < e1) {
        const int m = (e0 + e1) >> 1;
        if (__ldg(col + m) < key) e0 = m + 1;
        else e1 = m;
    }
    return e0;
}
// the cells of columns jb .. jb+3 of `row` with amplitude a (the cluster kernel stages
// its amplitudes in shared memory, so this form takes the value)
__device__ __forceinline__ void apply_cells_a(const mtb_cells &cl, int row, float a, int jb,
                                              float (&v)[4]) {
    if (cl.n == 0 || row < cl.row_lo || row > cl.row_hi) return;
    const int e0 = __ldg(cl.row_ptr + row), e1 = __ldg(cl.row_ptr + row + 1);
    if (e0 == e1) return;
    for (int e = lower_col(cl.col, e0, e1, jb); e < e1; ++e) {
        const int c = __ldg(cl.col + e) - jb;
        if (c >= 4) break;
        const float w = __ldg(cl.w + e);
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (c == q) v[q] -= a * w;
    }
}
__device__ __forceinline__ void apply_cells(const mtb_cells &cl, int row, const float *amp,
                                            int jb, float (&v)[4]) {
    if (cl.n == 0 || row < cl.row_lo || row > cl.row_hi) return;
    const int e0 = __ldg(cl.row_ptr + row), e1 = __ldg(cl.row_ptr + row + 1);
    if (e0 == e1) return;
    const float a = __ldg(amp + cl.amp_col);
    // only the cells of columns jb .. jb+3, in list order (duplicates included)
    for (int e = lower_col(cl.col, e0, e1, jb); e < e1; ++e) {
        const int c = __ldg(cl.col + e) - jb;
        if (c >= 4) break;
        const float w = __ldg(cl.w + e);
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (c == q) v[q] -= a * w;
    }
}
__device__ __forceinline__ float apply_cell1(const mtb_cells &cl, int row, int col,
                                             const float *amp, float v) {
    if (cl.n == 0 || row < cl.row_lo || row > cl.row_hi) return v;
    const int e0 = __ldg(cl.row_ptr + row), e1 = __ldg(cl.row_ptr + row + 1);
    if (e0 == e1) return v;
    const float a = __ldg(amp + cl.amp_col);
    for (int e = lower_col(cl.col, e0, e1, col); e < e1 && __ldg(cl.col + e) == col; ++e)
        v -= a * __ldg(cl.w + e);
    return v;
}

// Copy this row's values of component `comp` into the (pre-filtered) line samples.
__device__ __forceinline__ void sample_row(const mtb_line_sample *L, int nl, int comp, int i,
                                           int jb, bool act, const float (&v)[4], float *ring) {
    if (!act) return;
    for (int l = 0; l < nl; ++l) {
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

// ------------------------------------------------------------------ TM
// Column validity is folded into per-lane step coefficients (dt/dx times a
// 0/1 mask): a masked cell is left unchanged and box padding (where 1/eps is
// 0) stays zero, so the row body carries no per-element predicates. CPML
// memory is touched only on x-layer rows (row-uniform branch) and in y-layer
// lanes (bit masks, bit q = column jb+q), where the profiles are read from L1.
#define BIT(m, q) (((m) >> (q)) & 1u)

template <bool EXPL>
__device__ __forceinline__ void tm_warp(const mtb_yee2d_struct &S, const int i0, const int i1,
                                        const int c0, const Ctx2D &C, const mtb_line_sample *L,
                                        const int nl, Pipe<4> pp) {
    const int lane = threadIdx.x & 31;
    const int nx = S.nx, ny = S.ny;
    const int64_t P = S.pitch;
    const int jb = c0 + 4 * lane;
    const bool act = jb < S.pitch;
    const float dt = S.dt;
    const float rdx = 1.0f / S.dx;
    const float kdt = dt * rdx;
    const int par = C.par;
    float *__restrict__ Dzn = S.f_main[par ^ 1];
    float *__restrict__ Hxn = S.f_x[par ^ 1];
    float *__restrict__ Hyn = S.f_y[par ^ 1];
    float *ring = C.ring;
    const int64_t rf0 = S.ring_full[0], rf1 = S.ring_full[1], rf2 = S.ring_full[2];
    const int xb0 = S.xband[0], xb1 = S.xband[1], xe0 = S.xband[2], xe1 = S.xband[3];
    const int selo = S.src_e.row_lo, sehi = S.src_e.row_hi;
    const int h1lo = S.src_h1.row_lo, h1hi = S.src_h1.row_hi;
    const int h2lo = S.src_h2.row_lo, h2hi = S.src_h2.row_hi;

    // staged arrays: 0 Dz, 1 1/eps, 2 Hx, 3 Hy
    if (lane == 0) {
        const float **sp = const_cast<const float **>(pp.src);
        sp[0] = S.f_main[par];
        sp[1] = S.inv_eps_a;
        sp[2] = S.f_x[par];
        sp[3] = S.f_y[par];
    }
    __syncwarp();

    float kH[4], kD[4];                    // dt/dx on live Hx / Dz columns, else 0
    unsigned hyA = 0, eyA = 0;             // y-layer columns of this lane
    {
        const bool pmc = S.y_pmc != 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = jb + q;
            const bool hx = j <= ny - 2;
            const bool dz = pmc ? (j < ny) : (j >= 1 && j <= ny - 2);
            kH[q] = hx ? kdt : 0.f;
            kD[q] = dz ? kdt : 0.f;
            if (act && hx && (__ldg(S.hy_a + j) != 0.f || __ldg(S.hy_b + j) != 1.f)) hyA |= 1u << q;
            if (act && dz && (__ldg(S.ey_a + j) != 0.f || __ldg(S.ey_b + j) != 1.f)) eyA |= 1u << q;
        }
    }
    // halo columns: c0-1 (left of lane 0) and c0+128 (right of lane 31); the
    // halo values are computed by the whole warp (uniform) and selected
    const int jl = c0 - 1;
    const bool hasL = jl >= 0 && jl <= ny - 2;
    const bool hyAL = hasL && (__ldg(S.hy_a + jl) != 0.f || __ldg(S.hy_b + jl) != 1.f);
    const int jr = c0 + 128;
    const int so = 4 + 4 * lane;           // lane offset in a staged row

    // Ez = Dz / eps of staged row k (own 4, halos c0-1, c0+128)
    auto ez_of = [&](int k, int r, float (&ez)[4], float &ezl, float &ezr) {
        ezl = ezr = 0.f;
        if (r < 0 || r >= nx) { zero4(ez); return; }
        if (EXPL) {
            const float *Eex = S.e_explicit;
            if (act) ld4(Eex + r * P + jb, ez); else zero4(ez);
            if (jl >= 0) ezl = Eex[r * P + jl];
            if (jr < ny) ezr = Eex[r * P + jr];
            return;
        }
        const float *dz = pp.row(k, 0), *ie = pp.row(k, 1);
        float d[4], e[4];
        lds4(dz + so, d);
        lds4(ie + so, e);
#pragma unroll
        for (int q = 0; q < 4; ++q) ez[q] = d[q] * e[q];
        if (!act) zero4(ez);
        if (jl >= 0) ezl = dz[3] * ie[3];
        if (jr < ny) ezr = dz[132] * ie[132];
    };
    // Hy(n+1/2) of row r from Ez rows r (ea), r+1 (eb) (core/stepper_tm.py:97-100, :119-128)
    auto hy_new = [&](int k, int r, const float (&ea)[4], const float (&eb)[4], float (&out)[4],
                      bool own) {
        if (r < 0 || r >= nx) { zero4(out); return; }
        lds4(pp.row(k, 3) + so, out);
        if (r > nx - 2) return;                       // padding row of the box
        if (r >= xb0 && r < xb1) {
#pragma unroll
            for (int q = 0; q < 4; ++q) out[q] = fmaf(kdt, eb[q] - ea[q], out[q]);
        } else if (act) {                             // inside the x layer
            const float b = __ldg(S.hx_b + r), a = __ldg(S.hx_a + r);
            const int64_t o = r * P + jb;
            float ps[4];
            ld4(S.psi[1][par] + o, ps);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float d = (eb[q] - ea[q]) * rdx;
                ps[q] = b * ps[q] + a * d;
                out[q] = out[q] + dt * (d + ps[q]);
            }
            if (own) st4(S.psi[1][par ^ 1] + o, ps);
        }
        if (r >= h1lo && r <= h1hi && act) apply_cells(S.src_h1, r, C.amp_h, jb, out);
    };

    // ---- prologue: rows i0-1 (stage 0) and i0 (stage 1)
    for (int k = 0; k < NST; ++k) pp.issue(k);
    if (!pp.wait(0, C.err) || !pp.wait(1, C.err)) { pp.drain(0, NST); return; }
    float ezB[4], hyP[4], ezLB, ezRB;
    {
        float ezA[4], l, r;
        ez_of(0, i0 - 1, ezA, l, r);
        ez_of(1, i0, ezB, ezLB, ezRB);
        if (i0 >= 1) hy_new(0, i0 - 1, ezA, ezB, hyP, false); else zero4(hyP);
    }
    __syncwarp();
    pp.issue(NST);                          // stage 0 is free

    for (int i = i0; i < i1; ++i) {
        const int kc = i - i0 + 1, kn = kc + 1;
        if (!pp.wait(kn, C.err)) { pp.drain(kn + 1, kc + NST); return; }
        float ezC[4], ezLC, ezRC;
        ez_of(kn, i + 1, ezC, ezLC, ezRC);
        const int64_t ro = i * P + jb;

        float hyN[4];
        hy_new(kc, i, ezB, ezC, hyN, true);

        // Hx(n+1/2), row i (core/stepper_tm.py:91-94, :121-128)
        float hxN[4];
        const float *hxs = pp.row(kc, 2);
        float ezr = __shfl_down_sync(0xffffffffu, ezB[0], 1);
        ezr = (lane == 31) ? ezRB : ezr;
        lds4(hxs + so, hxN);
        if (!hyA) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float er = (q < 3) ? ezB[q + 1] : ezr;
                hxN[q] = fmaf(-kH[q], er - ezB[q], hxN[q]);
            }
        } else {
            float ps[4];
            ld4(S.psi[0][par] + ro, ps);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float er = (q < 3) ? ezB[q + 1] : ezr;
                const float d = (er - ezB[q]) * rdx;
                float c = d;
                if (BIT(hyA, q)) {
                    ps[q] = __ldg(S.hy_b + jb + q) * ps[q] + __ldg(S.hy_a + jb + q) * d;
                    c = d + ps[q];
                }
                hxN[q] = kH[q] != 0.f ? hxN[q] - dt * c : hxN[q];
            }
            st4(S.psi[0][par ^ 1] + ro, ps);
        }
        if (i >= h2lo && i <= h2hi && act) apply_cells(S.src_h2, i, C.amp_h, jb, hxN);
        if (!act) zero4(hxN);
        // left neighbour Hx(n+1/2)(i, j-1): lane 0's is the halo column,
        // recomputed by the whole warp from Ez(i, c0-1), Ez(i, c0)
        float hxl0 = __shfl_up_sync(0xffffffffu, hxN[3], 1);
        {
            const float ez0 = __shfl_sync(0xffffffffu, ezB[0], 0);
            float v = 0.f;
            if (hasL) {
                const float d = (ez0 - ezLB) * rdx;
                float c = d;
                if (hyAL)
                    c = d + (__ldg(S.hy_b + jl) * S.psi[0][par][i * P + jl] + __ldg(S.hy_a + jl) * d);
                v = hxs[3] - dt * c;
                if (i >= h2lo && i <= h2hi) v = apply_cell1(S.src_h2, i, jl, C.amp_h, v);
            }
            hxl0 = (lane == 0) ? v : hxl0;
        }

        // Dz(n+1), row i (core/stepper_tm.py:136-166), then source and E
        float dzN[4], ezN[4], ieB[4];
        lds4(pp.row(kc, 0) + so, dzN);
        lds4(pp.row(kc, 1) + so, ieB);
        if (i >= 1 && i <= nx - 2) {
            const bool pxA = act && (i < xe0 || i >= xe1);
            if (!pxA && !eyA) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float hxm = (q == 0) ? hxl0 : hxN[q - 1];
                    dzN[q] = fmaf(kD[q], (hyN[q] - hyP[q]) - (hxN[q] - hxm), dzN[q]);
                }
            } else {
                float bx = 1.f, ax = 0.f;
                if (pxA) { bx = __ldg(S.ex_b + i); ax = __ldg(S.ex_a + i); }
                float px[4], py[4];
                if (pxA) ld4(S.psi[2][par] + ro, px); else zero4(px);
                if (eyA) ld4(S.psi[3][par] + ro, py); else zero4(py);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (kD[q] == 0.f) continue;
                    const float hxm = (q == 0) ? hxl0 : hxN[q - 1];
                    const float dhy = (hyN[q] - hyP[q]) * rdx;
                    const float dhx = (hxN[q] - hxm) * rdx;
                    float p1 = 0.f, p2 = 0.f;
                    if (pxA) { p1 = bx * px[q] + ax * dhy; px[q] = p1; }
                    if (BIT(eyA, q)) {
                        p2 = __ldg(S.ey_b + jb + q) * py[q] + __ldg(S.ey_a + jb + q) * dhx;
                        py[q] = p2;
                    }
                    dzN[q] = dzN[q] + dt * (((dhy + p1) - dhx) - p2);
                }
                if (pxA) st4(S.psi[2][par ^ 1] + ro, px);
                if (eyA) st4(S.psi[3][par ^ 1] + ro, py);
            }
        }
        if (i >= selo && i <= sehi && act) apply_cells(S.src_e, i, C.amp_e, jb, dzN);
#pragma unroll
        for (int q = 0; q < 4; ++q) ezN[q] = dzN[q] * ieB[q];
        if (act) {
            st4(Hxn + ro, hxN);
            st4(Hyn + ro, hyN);
            st4(Dzn + ro, dzN);
            if (rf0 >= 0) st4(ring + rf0 + ro, ezN);
            if (rf1 >= 0) st4(ring + rf1 + ro, hxN);
            if (rf2 >= 0) st4(ring + rf2 + ro, hyN);
        }
        if (nl) {
            sample_row(L, nl, MTB_C2_MAIN, i, jb, act, ezN, ring);
            sample_row(L, nl, MTB_C2_X, i, jb, act, hxN, ring);
            sample_row(L, nl, MTB_C2_Y, i, jb, act, hyN, ring);
        }
        copy4(hyP, hyN);
        copy4(ezB, ezC);
        ezLB = ezLC;
        ezRB = ezRC;
        __syncwarp();
        pp.issue(kc + NST);                   // row i's stage is free
    }
}

// ------------------------------------------------------------------ TE

__device__ __forceinline__ void te_warp(const mtb_yee2d_struct &S, const int i0, const int i1,
                                        const int c0, const Ctx2D &C, const mtb_line_sample *L,
                                        const int nl, Pipe<5> pp) {
    const int lane = threadIdx.x & 31;
    const int nx = S.nx, ny = S.ny;
    const int64_t P = S.pitch;
    const int jb = c0 + 4 * lane;
    const bool act = jb < S.pitch;
    const float dt = S.dt;
    const float rdx = 1.0f / S.dx;
    const float kdt = dt * rdx;
    const int par = C.par;
    float *__restrict__ Hzn = S.f_main[par ^ 1];
    float *__restrict__ Dxn = S.f_x[par ^ 1];
    float *__restrict__ Dyn = S.f_y[par ^ 1];
    float *ring = C.ring;
    const int64_t rf0 = S.ring_full[0], rf1 = S.ring_full[1], rf2 = S.ring_full[2];
    const int xb0 = S.xband[0], xb1 = S.xband[1], xe0 = S.xband[2], xe1 = S.xband[3];
    const int selo = S.src_e.row_lo, sehi = S.src_e.row_hi;
    const int h1lo = S.src_h1.row_lo, h1hi = S.src_h1.row_hi;

    // staged arrays: 0 Hz, 1 Dx, 2 Dy, 3 1/eps_x, 4 1/eps_y
    if (lane == 0) {
        const float **sp = const_cast<const float **>(pp.src);
        sp[0] = S.f_main[par];
        sp[1] = S.f_x[par];
        sp[2] = S.f_y[par];
        sp[3] = S.inv_eps_a;
        sp[4] = S.inv_eps_b;
    }
    __syncwarp();

    float kDx[4], kDy[4];                  // dt/dx on updated Dx / live Dy, Hz columns
    unsigned eyA = 0, hyA = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        const bool hz = j <= ny - 2, dxu = j >= 1 && j <= ny - 2;
        kDx[q] = dxu ? kdt : 0.f;
        kDy[q] = hz ? kdt : 0.f;           // Dy and Hz live on columns j <= ny-2
        if (act && dxu && (__ldg(S.ey_a + j) != 0.f || __ldg(S.ey_b + j) != 1.f)) eyA |= 1u << q;
        if (act && hz && (__ldg(S.hy_a + j) != 0.f || __ldg(S.hy_b + j) != 1.f)) hyA |= 1u << q;
    }
    const int jl = c0 - 1;          // left halo: Hz(r, c0-1)
    const int jr = c0 + 128;        // right halo: Ex(n+1/2)(r, c0+128), uniform
    const bool hasR = jr <= ny - 1;
    const bool updR = hasR && jr >= 1 && jr <= ny - 2;
    const bool eyAR = updR && (__ldg(S.ey_a + jr) != 0.f || __ldg(S.ey_b + jr) != 1.f);
    const int so = 4 + 4 * lane;

    // Hz(n) of staged row k (zero outside the Hz array)
    auto hz_of = [&](int k, int r, float (&v)[4], float &hl, float &hr) {
        hl = hr = 0.f;
        if (!(r >= 0 && r <= nx - 2)) { zero4(v); return; }
        const float *h = pp.row(k, 0);
        lds4(h + so, v);
        if (!act) zero4(v);
        if (jl >= 0 && jl <= ny - 2) hl = h[3];
        if (jr <= ny - 2) hr = h[132];
    };

    // D/E(n+1/2) of row r (stage k) from Hz(n) rows r-1 (hp) and r (hc)
    // (core/stepper_te.py:79-111 D update, :120-134 source, :150-175 E)
    auto e_row = [&](int k, int r, const float (&hp)[4], const float (&hc)[4], float hzL,
                     float hzR, bool own, float (&ex)[4], float (&ey)[4], float &exR) {
        exR = 0.f;
        if (r < 0 || r >= nx) { zero4(ex); zero4(ey); return; }
        const int64_t ro = r * P + jb;
        const float *sdx = pp.row(k, 1), *sdy = pp.row(k, 2), *siex = pp.row(k, 3),
                    *siey = pp.row(k, 4);
        float dxN[4];
        lds4(sdx + so, dxN);
        float hl = __shfl_up_sync(0xffffffffu, hc[3], 1);
        hl = (lane == 0) ? hzL : hl;
        if (r <= nx - 2) {
            if (!eyA) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float hm = (q == 0) ? hl : hc[q - 1];
                    dxN[q] = fmaf(kDx[q], hc[q] - hm, dxN[q]);
                }
            } else {
                float py[4];
                ld4(S.psi[0][par] + ro, py);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (kDx[q] == 0.f) continue;
                    const float hm = (q == 0) ? hl : hc[q - 1];
                    const float d = (hc[q] - hm) * rdx;
                    float c = d;
                    if (BIT(eyA, q)) {
                        py[q] = __ldg(S.ey_b + jb + q) * py[q] + __ldg(S.ey_a + jb + q) * d;
                        c = d + py[q];
                    }
                    dxN[q] = dxN[q] + dt * c;
                }
                if (own) st4(S.psi[0][par ^ 1] + ro, py);
            }
            float ie[4];
            lds4(siex + so, ie);
#pragma unroll
            for (int q = 0; q < 4; ++q) ex[q] = dxN[q] * ie[q];
            if (hasR) {
                float dxr = sdx[132];
                if (updR) {
                    const float hc127 = __shfl_sync(0xffffffffu, hc[3], 31);
                    const float d = (hzR - hc127) * rdx;
                    float c = d;
                    if (eyAR)
                        c = d + (__ldg(S.ey_b + jr) * S.psi[0][par][r * P + jr] +
                                 __ldg(S.ey_a + jr) * d);
                    dxr = dxr + dt * c;
                }
                exR = dxr * siex[132];
            }
        } else {
            zero4(ex);
        }
        float dyN[4];
        lds4(sdy + so, dyN);
        if (r >= 1 && r <= nx - 2) {
            if (!(act && (r < xe0 || r >= xe1))) {
#pragma unroll
                for (int q = 0; q < 4; ++q) dyN[q] = fmaf(-kDy[q], hc[q] - hp[q], dyN[q]);
            } else {
                const float bx = __ldg(S.ex_b + r), ax = __ldg(S.ex_a + r);
                float px[4];
                ld4(S.psi[1][par] + ro, px);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (kDy[q] == 0.f) continue;
                    const float d = (hc[q] - hp[q]) * rdx;
                    px[q] = bx * px[q] + ax * d;
                    dyN[q] = dyN[q] - dt * (d + px[q]);
                }
                if (own) st4(S.psi[1][par ^ 1] + ro, px);
            }
        }
        if (r >= selo && r <= sehi && act) apply_cells(S.src_e, r, C.amp_e, jb, dyN);
        float ie[4];
        lds4(siey + so, ie);
#pragma unroll
        for (int q = 0; q < 4; ++q) ey[q] = dyN[q] * ie[q];
        if (!act) { zero4(ex); zero4(ey); }
        if (own && act) {
            st4(Dxn + ro, dxN);
            st4(Dyn + ro, dyN);
            if (rf1 >= 0) st4(ring + rf1 + ro, ex);
            if (rf2 >= 0) st4(ring + rf2 + ro, ey);
        }
        if (own && nl) {
            sample_row(L, nl, MTB_C2_X, r, jb, act, ex, ring);
            sample_row(L, nl, MTB_C2_Y, r, jb, act, ey, ring);
        }
    };

    // ---- prologue: rows i0-1 (stage 0), i0 (stage 1)
    for (int k = 0; k < NST; ++k) pp.issue(k);
    if (!pp.wait(0, C.err) || !pp.wait(1, C.err)) { pp.drain(0, NST); return; }
    float hzB[4], exB[4], eyB[4], exRB;
    {
        float hzA[4], l0, r0, lB, rB;
        hz_of(0, i0 - 1, hzA, l0, r0);
        hz_of(1, i0, hzB, lB, rB);
        e_row(1, i0, hzA, hzB, lB, rB, true, exB, eyB, exRB);
    }
    __syncwarp();
    pp.issue(NST);

    for (int i = i0; i < i1; ++i) {
        const int kc = i - i0 + 1, kn = kc + 1;
        if (!pp.wait(kn, C.err)) { pp.drain(kn + 1, kc + NST); return; }
        float hzC[4], exC[4], eyC[4], exRC, lC, rC;
        hz_of(kn, i + 1, hzC, lC, rC);
        e_row(kn, i + 1, hzB, hzC, lC, rC, i + 1 < i1, exC, eyC, exRC);

        // Hz(n+1), row i (core/stepper_te.py:113-117)
        const int64_t ro = i * P + jb;
        float hzN[4];
        copy4(hzN, hzB);
        if (i <= nx - 2) {
            float exr = __shfl_down_sync(0xffffffffu, exB[0], 1);
            exr = (lane == 31) ? exRB : exr;
            const bool pxA = act && (i < xb0 || i >= xb1);
            if (!pxA && !hyA) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float exn = (q < 3) ? exB[q + 1] : exr;
                    hzN[q] = fmaf(-kDy[q], (eyC[q] - eyB[q]) - (exn - exB[q]), hzN[q]);
                }
            } else {
                float bx = 1.f, ax = 0.f;
                if (pxA) { bx = __ldg(S.hx_b + i); ax = __ldg(S.hx_a + i); }
                float p1v[4], p2v[4];
                if (pxA) ld4(S.psi[2][par] + ro, p1v); else zero4(p1v);
                if (hyA) ld4(S.psi[3][par] + ro, p2v); else zero4(p2v);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (kDy[q] == 0.f) continue;
                    const float exn = (q < 3) ? exB[q + 1] : exr;
                    const float dey = (eyC[q] - eyB[q]) * rdx;
                    const float dex = (exn - exB[q]) * rdx;
                    float p1 = 0.f, p2 = 0.f;
                    if (pxA) { p1 = bx * p1v[q] + ax * dey; p1v[q] = p1; }
                    if (BIT(hyA, q)) {
                        p2 = __ldg(S.hy_b + jb + q) * p2v[q] + __ldg(S.hy_a + jb + q) * dex;
                        p2v[q] = p2;
                    }
                    hzN[q] = hzN[q] - dt * (((dey + p1) - dex) - p2);
                }
                if (pxA) st4(S.psi[2][par ^ 1] + ro, p1v);
                if (hyA) st4(S.psi[3][par ^ 1] + ro, p2v);
            }
            if (i >= h1lo && i <= h1hi && act) apply_cells(S.src_h1, i, C.amp_h, jb, hzN);
        }
        if (act) {
            st4(Hzn + ro, hzN);
            if (rf0 >= 0) st4(ring + rf0 + ro, hzN);
        }
        if (nl) sample_row(L, nl, MTB_C2_MAIN, i, jb, act, hzN, ring);
        copy4(hzB, hzC);
        copy4(exB, exC);
        copy4(eyB, eyC);
        exRB = exRC;
        __syncwarp();
        pp.issue(kc + NST);
    }
}

// Shared memory per block: per warp its NST staged rows (first: bulk-copy
// destinations need 16-byte alignment), its mbarriers, its structure copy and
// its filtered line samples.
template <int NA>
struct __align__(16) WarpSmem {
    float buf[NST * NA * EXT];
    uint64_t bar[NST];
    const float *src[8];
    mtb_yee2d_struct s;
    mtb_line_sample lines[MAXL];
};
static_assert((NST * 4 * EXT * sizeof(float)) % 16 == 0, "stage buffers must be 16-byte aligned");
static_assert(sizeof(WarpSmem<4>) % 16 == 0 && sizeof(WarpSmem<5>) % 16 == 0,
              "per-warp shared block must keep 16-byte alignment");

// Per-warp setup shared by the TM and TE kernels: descriptor copy, barrier
// init, line-sample filter, pipeline geometry.
template <int NA>
__device__ __forceinline__ bool warp_setup(const mtb_yee2d_struct *__restrict__ SS,
                                           const int4 *__restrict__ work, int n_work,
                                           WarpSmem<NA> *&Wp, int4 &w, int &nl) {
    extern __shared__ __align__(16) unsigned char smraw[];
    WarpSmem<NA> *ws = reinterpret_cast<WarpSmem<NA> *>(smraw);
    const int wib = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int wid = blockIdx.x * WARPS2D + wib;
    if (wid >= n_work) return false;             // whole warp
    WarpSmem<NA> &W = ws[wib];
    Wp = &W;
    w = work[wid];
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(SS + w.x);
        uint32_t *dst = reinterpret_cast<uint32_t *>(&W.s);
        for (int e = lane; e < (int)(sizeof(mtb_yee2d_struct) / 4); e += 32) dst[e] = src[e];
    }
    if (lane == 0) {
        for (int k = 0; k < NST; ++k) mbar_init(&W.bar[k], 1);
        mbar_fence_init();
    }
    __syncwarp();
    const mtb_yee2d_struct &S = W.s;
    const int i0 = w.y, i1 = w.z, c0 = w.w;
    {   // line samples that touch this warp's rows [i0, i1) x columns [c0, c0+128)
        const int n_all = S.n_lines;
        bool keep = false;
        mtb_line_sample ln{};
        if (lane < n_all) {
            ln = S.lines[lane];
            if (ln.kind == 0)
                keep = ln.index >= i0 && ln.index < i1 && ln.lo < c0 + 128 && ln.hi > c0;
            else
                keep = ln.index >= c0 && ln.index < c0 + 128 && ln.lo < i1 && ln.hi > i0;
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) W.lines[__popc(m & ((1u << lane) - 1))] = ln;
        nl = __popc(m);
    }
    __syncwarp();
    return true;
}

template <int NA>
__device__ __forceinline__ Pipe<NA> make_pipe(WarpSmem<NA> &W, int i0, int i1, int c0) {
    Pipe<NA> pp;
    const mtb_yee2d_struct &S = W.s;
    pp.buf = W.buf;
    pp.bar = W.bar;
    pp.src = W.src;
    pp.P = S.pitch;
    pp.w0 = max(c0 - 4, 0);
    const int w1 = min(c0 + 132, S.pitch);
    pp.dst = pp.w0 - (c0 - 4);
    pp.bytes = (uint32_t)(w1 - pp.w0) * 4u;
    pp.i0m1 = i0 - 1;
    pp.nx = S.nx;
    pp.nrows = i1 - i0 + 2;
    pp.lane = threadIdx.x & 31;
    return pp;
}

// TM step; FIRST = the plan's first step, where a structure imported with an
// Ez that is not Dz/eps reads it from e_explicit.
template <bool FIRST>
__global__ void __launch_bounds__(32 * WARPS2D, 4) k_yee2d_tm(
    const mtb_yee2d_struct *__restrict__ SS, const int4 *__restrict__ work, int n_work,
    Ctx2D C) {
    WarpSmem<4> *W;
    int4 w;
    int nl;
    if (!warp_setup<4>(SS, work, n_work, W, w, nl)) return;
    Pipe<4> pp = make_pipe<4>(*W, w.y, w.z, w.w);
    if (FIRST && W->s.explicit_e)
        tm_warp<true>(W->s, w.y, w.z, w.w, C, W->lines, nl, pp);
    else
        tm_warp<false>(W->s, w.y, w.z, w.w, C, W->lines, nl, pp);
}

__global__ void __launch_bounds__(32 * WARPS2D, 4) k_yee2d_te(
    const mtb_yee2d_struct *__restrict__ SS, const int4 *__restrict__ work, int n_work,
    Ctx2D C) {
    WarpSmem<5> *W;
    int4 w;
    int nl;
    if (!warp_setup<5>(SS, work, n_work, W, w, nl)) return;
    Pipe<5> pp = make_pipe<5>(*W, w.y, w.z, w.w);
    te_warp(W->s, w.y, w.z, w.w, C, W->lines, nl, pp);
}

// ================================================================== tiles
// Tile kernels: a block owns TROWS rows x 128 columns of one structure;
// thread (lane, row) updates one float4 (columns jb .. jb+3) of one row and
// issues every load it needs before using any. The one-row / one-column
// halos of the fused step are recomputed from the old state (hence the
// ping-pong buffers); neighbouring rows come from L1/L2, neighbouring columns
// from warp shuffles (lane 0 and lane 31 load their outer column). The CPML
// memory is gated by the plan's band limits (geometry); inside a band the
// recursion runs with the profile's (b, a), which are (1, 0) on inert nodes,
// so lanes of one warp run the same arithmetic whether or not they are in a
// layer, and the edge rules are selects.
constexpr int TROWS = 8;            // warps per tile block
constexpr int WROWS = 4;            // rows per warp
constexpr int TILE_ROWS = TROWS * WROWS;
// tile blocks (of WROWS rows per warp) below which the tiles use one row per
// warp: 148 SMs x 2 resident blocks x 4 waves
constexpr int64_t TILE_MIN_BLOCKS = 148 * 2 * 4;

struct TileSmem {
    mtb_yee2d_struct s;
    mtb_line_sample lines[MAXL];
    int nl;
};

// Block setup: work item, structure copy, line samples touching the tile.
__device__ __forceinline__ bool tile_setup(const mtb_yee2d_struct *__restrict__ SS,
                                           const int4 *__restrict__ work, int n_work, int wr,
                                           TileSmem &T, int4 &w) {
    if ((int)blockIdx.x >= n_work) return false;
    w = __ldg(work + blockIdx.x);
    const int tid = threadIdx.y * 32 + threadIdx.x;
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(SS + w.x);
        uint32_t *dst = reinterpret_cast<uint32_t *>(&T.s);
        for (int e = tid; e < (int)(sizeof(mtb_yee2d_struct) / 4); e += 32 * TROWS)
            dst[e] = __ldg(src + e);
    }
    __syncthreads();
    if (threadIdx.y == 0) {
        const int i0 = w.y, i1 = min(w.y + TROWS * wr, T.s.nx), c0 = w.z;
        const int n_all = T.s.n_lines;
        bool keep = false;
        mtb_line_sample ln{};
        if (threadIdx.x < n_all) {
            ln = T.s.lines[threadIdx.x];
            if (ln.kind == 0)
                keep = ln.index >= i0 && ln.index < i1 && ln.lo < c0 + 128 && ln.hi > c0;
            else
                keep = ln.index >= c0 && ln.index < c0 + 128 && ln.lo < i1 && ln.hi > i0;
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) T.lines[__popc(m & ((1u << threadIdx.x) - 1))] = ln;
        if (threadIdx.x == 0) T.nl = __popc(m);
    }
    __syncthreads();
    return true;
}

__device__ __forceinline__ bool in_band(int k, int lo, int hi) { return k < lo || k >= hi; }
// any of columns jb .. jb+3 in a band
__device__ __forceinline__ bool band4(int jb, int lo, int hi) { return jb < lo || jb + 3 >= hi; }

// Hy(n+1/2) of one row from Ez rows r (ea), r+1 (eb): core/stepper_tm.py:97-100,
// :119-128, magnetic sheet source :116-118. `valid` = r <= nx-2.
// With magnetic conductivity / permeability (`h1`, `h2` non-null, box layout):
// Hy' = h1 Hy + h2 curl (core/stepper_tm.py:121-125).
__device__ __forceinline__ void tm_hy(const mtb_yee2d_struct &S, int r, bool valid, bool act,
                                      int jb, float b, float a, float dt, float rdx,
                                      const float (&ea)[4], const float (&eb)[4],
                                      const float (&hy)[4], float (&ps)[4], float (&out)[4],
                                      const float *amp_h, const float *h1 = nullptr,
                                      const float *h2 = nullptr) {
    float m1[4] = {1.f, 1.f, 1.f, 1.f}, m2[4] = {dt, dt, dt, dt};
    if (h1 && valid && act) {
        const uint32_t o = (uint32_t)r * S.pitch + jb;
        ld4(h1 + o, m1);
        ld4(h2 + o, m2);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float d = (eb[q] - ea[q]) * rdx;
        const float pv = b * ps[q] + a * d;
        const float hn = h1 ? m1[q] * hy[q] + m2[q] * (d + pv) : hy[q] + dt * (d + pv);
        out[q] = valid ? hn : hy[q];
        ps[q] = valid ? pv : ps[q];
    }
    if (valid && act && r >= S.src_h1.row_lo && r <= S.src_h1.row_hi)
        apply_cells(S.src_h1, r, amp_h, jb, out);
}

// Instantaneous chi2 / chi3 (core/stepper_tm.py:222-230): Ez = rhs / eps, then three
// sweeps Ez = rhs / (eps + chi2 Ez + chi3 Ez Ez), evaluated left to right and rounded
// like the reference's tensor expression.
__device__ __forceinline__ float tm_nl(float rhs, float eps, float x2, float x3) {
    float e = __fdiv_rn(rhs, eps);
#pragma unroll
    for (int k = 0; k < 3; ++k)
        e = __fdiv_rn(rhs, __fadd_rn(__fadd_rn(eps, __fmul_rn(x2, e)),
                                     __fmul_rn(__fmul_rn(x3, e), e)));
    return e;
}

// Ez of one row's float4 from rhs = Dz - sum P: rhs / eps (as rhs * (1/eps)), or the
// chi2 / chi3 fixed point when the structure has them (box offset o).
__device__ __forceinline__ void tm_e4(const mtb_yee2d_struct &S, bool nl, uint32_t o,
                                      const float (&rhs)[4], const float (&ie)[4],
                                      float (&e)[4]) {
    if (nl) {
        float x2[4], x3[4], ep[4];
        ld4(S.chi2 + o, x2);
        ld4(S.chi3 + o, x3);
        ld4(S.eps_nl + o, ep);
#pragma unroll
        for (int q = 0; q < 4; ++q) e[q] = tm_nl(rhs[q], ep[q], x2[q], x3[q]);
    } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) e[q] = rhs[q] * ie[q];
    }
}

// Ez(n) of one cell as tm_tile forms it for its own rows: the imported Ez on an
// explicit first step, else (Dz - sum_k P_k) / eps with the poles summed in order.
template <bool EXPL, bool EXT>
__device__ __forceinline__ float tm_ez_at(const mtb_yee2d_struct &S, const Ctx2D &C, int i,
                                          int j) {
    const uint32_t o = (uint32_t)i * S.pitch + j;
    if (EXPL) return S.e_explicit[o];
    float sp = 0.f;
    const float *Pc = S.pol_p[C.pst];
    const uint32_t pl = (uint32_t)S.nx * S.pitch;
#pragma unroll 1
    for (int k = 0; k < (EXT ? S.n_poles : 0); ++k) sp += Pc[k * pl + o];
    if (EXT && S.chi2)
        return tm_nl(S.f_main[C.par][o] - sp, S.eps_nl[o], S.chi2[o], S.chi3[o]);
    return (S.f_main[C.par][o] - sp) * S.inv_eps_a[o];
}

// The live on-plane H line beyond a TM symmetry cut (core/stepper_tm.py:95-113):
// H0' = H0 -/+ dt (Ez_cut - ghost) / dx, ghost = ph * Ez(partner). `a` = 0 for
// the Hx row at the y cut (cell (k, 0), minus), 1 for the Hy column at the x cut
// (cell (0, k), plus); ez is Ez(n) of the cut cell.
template <bool EXPL, bool EXT>
__device__ __forceinline__ float tm_cut_line(const mtb_yee2d_struct &S, const Ctx2D &C, int a,
                                             int k, float ez, float dt, float rdx) {
    const int map = a ? S.cut_map_x : S.cut_map_y;
    const float ph = a ? S.cut_ph_x : S.cut_ph_y;
    float partner = ez;
    if (map == 1) partner = tm_ez_at<EXPL, EXT>(S, C, S.nx - 1 - k, 0);
    else if (map == 2) partner = a ? tm_ez_at<EXPL, EXT>(S, C, k, 0)
                                   : tm_ez_at<EXPL, EXT>(S, C, 0, k);
    const float d = (ez - ph * partner) * rdx;
    const float *h0 = a ? S.f_y0[C.par] : S.f_x0[C.par];
    return a ? h0[k] + dt * d : h0[k] - dt * d;
}

// Magnetic Lorentz poles on one float4 of an H row (core/stepper_tm.py:209-219): `bh`
// holds B(n+1/2) (the curl update and the sheet sources applied to B) and becomes
// H(n+1/2) = B - sum_k M_k(n+1), M(n+1) = mc1 M(n) + mc2 M(n-1) + mc3 H(n-1/2) (`hold`).
// `store` writes B and the M(n+1) stack (own rows; a recomputed halo row does not).
__device__ __forceinline__ void tm_mpole4(const mtb_yee2d_struct &S, const Ctx2D &C, int c,
                                          uint32_t o, bool store, const float (&hold)[4],
                                          float (&bh)[4]) {
    const uint32_t pl = (uint32_t)S.nx * S.pitch;
    const float *Mc = S.mpol[c][C.pst], *Mp = S.mpol[c][(C.pst + 2) % 3];
    float *Mo = S.mpol[c][(C.pst + 1) % 3];
    float sm[4];
    zero4(sm);
#pragma unroll 1
    for (int k = 0; k < S.n_mpoles; ++k) {
        const uint32_t ok = k * pl + o;
        float mc[4], mp[4], a1[4], a2[4], a3[4];
        ld4(Mc + ok, mc);
        ld4(Mp + ok, mp);
        ld4(S.mpc[c][0] + ok, a1);
        ld4(S.mpc[c][1] + ok, a2);
        ld4(S.mpc[c][2] + ok, a3);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            mc[q] = a1[q] * mc[q] + a2[q] * mp[q] + a3[q] * hold[q];
            sm[q] += mc[q];
        }
        if (store) st4(Mo + ok, mc);
    }
    if (store) st4(S.f_b[c][C.par ^ 1] + o, bh);
#pragma unroll
    for (int q = 0; q < 4; ++q) bh[q] = bh[q] - sm[q];
}

// The same for one cell (lane 0's recomputed left neighbour), not stored.
__device__ __forceinline__ float tm_mpole1(const mtb_yee2d_struct &S, const Ctx2D &C, int c,
                                           uint32_t o, float hold, float b) {
    const uint32_t pl = (uint32_t)S.nx * S.pitch;
    const float *Mc = S.mpol[c][C.pst], *Mp = S.mpol[c][(C.pst + 2) % 3];
    float sm = 0.f;
#pragma unroll 1
    for (int k = 0; k < S.n_mpoles; ++k) {
        const uint32_t ok = k * pl + o;
        sm += S.mpc[c][0][ok] * Mc[ok] + S.mpc[c][1][ok] * Mp[ok] + S.mpc[c][2][ok] * hold;
    }
    return b - sm;
}

template <bool EXPL, bool EXT, bool MP = false>
__device__ __forceinline__ void tm_tile(const mtb_yee2d_struct &S, const int i, const int c0,
                                        const Ctx2D &C, const mtb_line_sample *L, const int nl) {
    const int lane = threadIdx.x;
    const int nx = S.nx, ny = S.ny, P = S.pitch;
    const int jb = c0 + 4 * lane;
    const bool act = jb < P;
    const float dt = S.dt, rdx = 1.0f / S.dx;
    const int par = C.par;
    const uint32_t ro = (uint32_t)i * P + jb;        // box < 2^31 cells (plan check)
    const float *__restrict__ Dz = S.f_main[par];
    const float *__restrict__ Hx = S.f_x[par];
    const float *__restrict__ Hy = S.f_y[par];
    const float *__restrict__ ie = S.inv_eps_a;
    // symmetry cuts: the cut row (x) / column (y) of Dz is live
    const bool cutx = EXT && S.cut_x != 0, cuty = EXT && S.cut_y != 0;
    const bool hyRow = i <= nx - 2, dzRow = (i >= 1 || cutx) && i <= nx - 2;
    const bool bxH = hyRow && in_band(i, S.xband[0], S.xband[1]);
    const bool bxHp = i >= 1 && in_band(i - 1, S.xband[0], S.xband[1]);
    const bool bxE = dzRow && in_band(i, S.xband[2], S.xband[3]);
    const bool byH = act && band4(jb, S.yband[0], S.yband[1]);
    const bool byE = act && dzRow && band4(jb, S.yband[2], S.yband[3]);
    const int jl = jb - 1;
    const bool hasL = lane == 0 && jl >= 0 && jl <= ny - 2;
    const bool byHL = hasL && in_band(jl, S.yband[0], S.yband[1]);

    float ez0[4], ez1[4], ez2[4], d1[4], e1[4], hx[4], hy[4], hyp[4];
    float p0[4], p1[4], p1p[4], p2[4], p3[4];
    float ezl = 0.f, ezr = 0.f, hxl = 0.f, p0l = 0.f;
    zero4(ez0); zero4(ez1); zero4(ez2); zero4(d1); zero4(e1); zero4(hx); zero4(hy); zero4(hyp);
    zero4(p0); zero4(p1); zero4(p1p); zero4(p2); zero4(p3);
    if (act) {
        ld4(Dz + ro, d1);
        ld4(ie + ro, e1);
        if (EXPL) {
            const float *Eex = S.e_explicit;
            ld4(Eex + ro, ez1);
            if (i >= 1) ld4(Eex + ro - P, ez0);
            if (i + 1 < nx) ld4(Eex + ro + P, ez2);
            if (lane == 0 && jb >= 1) ezl = Eex[ro - 1];
            if (lane == 31 && jb + 4 < ny) ezr = Eex[ro + 4];
        } else {
            float d0[4], e0[4], d2[4], e2[4];
            zero4(d0); zero4(e0); zero4(d2); zero4(e2);
            if (i >= 1) { ld4(Dz + ro - P, d0); ld4(ie + ro - P, e0); }
            if (i + 1 < nx) { ld4(Dz + ro + P, d2); ld4(ie + ro + P, e2); }
            // dispersive poles: Ez = (Dz - sum_k P_k) / eps (core/stepper_tm.py:220-224)
            float s0[4], s1[4], s2[4], sl = 0.f, sr = 0.f;
            zero4(s0); zero4(s1); zero4(s2);
            const float *Pc = S.pol_p[C.pst];
            const uint32_t pl = (uint32_t)nx * P;
#pragma unroll 1
            for (int k = 0; k < (EXT ? S.n_poles : 0); ++k) {
                const float *Pk = Pc + k * pl;
                float t[4];
                ld4(Pk + ro, t);
#pragma unroll
                for (int q = 0; q < 4; ++q) s1[q] += t[q];
                if (i >= 1) {
                    ld4(Pk + ro - P, t);
#pragma unroll
                    for (int q = 0; q < 4; ++q) s0[q] += t[q];
                }
                if (i + 1 < nx) {
                    ld4(Pk + ro + P, t);
#pragma unroll
                    for (int q = 0; q < 4; ++q) s2[q] += t[q];
                }
                if (lane == 0 && jb >= 1) sl += Pk[ro - 1];
                if (lane == 31 && jb + 4 < P) sr += Pk[ro + 4];
            }
            const bool nl = EXT && S.chi2 != nullptr;
            if (lane == 0 && jb >= 1)
                ezl = nl ? tm_nl(Dz[ro - 1] - sl, S.eps_nl[ro - 1], S.chi2[ro - 1], S.chi3[ro - 1])
                         : (Dz[ro - 1] - sl) * ie[ro - 1];
            if (lane == 31 && jb + 4 < P)
                ezr = nl ? tm_nl(Dz[ro + 4] - sr, S.eps_nl[ro + 4], S.chi2[ro + 4], S.chi3[ro + 4])
                         : (Dz[ro + 4] - sr) * ie[ro + 4];
            float r0[4], r1[4], r2[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                r0[q] = d0[q] - s0[q];
                r1[q] = d1[q] - s1[q];
                r2[q] = d2[q] - s2[q];
            }
            if (i >= 1) tm_e4(S, nl, ro - P, r0, e0, ez0); else zero4(ez0);
            tm_e4(S, nl, ro, r1, e1, ez1);
            if (i + 1 < nx) tm_e4(S, nl, ro + P, r2, e2, ez2); else zero4(ez2);
        }
        ld4(Hx + ro, hx);
        ld4(Hy + ro, hy);
        if (i >= 1) ld4(Hy + ro - P, hyp);
        if (hasL) {
            hxl = Hx[ro - 1];
            if (byHL) p0l = S.psi[0][par][ro - 1];
        }
        if (byH) ld4(S.psi[0][par] + ro, p0);
        if (bxH) ld4(S.psi[1][par] + ro, p1);
        if (bxHp) ld4(S.psi[1][par] + ro - P, p1p);
        if (bxE) ld4(S.psi[2][par] + ro, p2);
        if (byE) ld4(S.psi[3][par] + ro, p3);
    }
    // profiles: (1, 0) outside the bands
    float hxb = 1.f, hxa = 0.f, hxbp = 1.f, hxap = 0.f, exb = 1.f, exa = 0.f;
    if (bxH) { hxb = __ldg(S.hx_b + i); hxa = __ldg(S.hx_a + i); }
    if (bxHp) { hxbp = __ldg(S.hx_b + i - 1); hxap = __ldg(S.hx_a + i - 1); }
    if (bxE) { exb = __ldg(S.ex_b + i); exa = __ldg(S.ex_a + i); }
    const bool pmc = S.y_pmc != 0;
    float hyb[4], hya[4], eyb[4], eya[4];
    bool vH[4], vD[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        vH[q] = act && j <= ny - 2;
        vD[q] = act && dzRow && (pmc ? (j < ny) : ((j >= 1 || cuty) && j <= ny - 2));
        const bool oh = byH && j <= ny - 2, oe = byE && j < ny;
        hyb[q] = oh ? __ldg(S.hy_b + j) : 1.f;
        hya[q] = oh ? __ldg(S.hy_a + j) : 0.f;
        eyb[q] = oe ? __ldg(S.ey_b + j) : 1.f;
        eya[q] = oe ? __ldg(S.ey_a + j) : 0.f;
    }
    float ezR = __shfl_down_sync(0xffffffffu, ez1[0], 1);
    if (lane == 31) ezR = ezr;

    // Hy(n+1/2) rows i-1 (recomputed halo) and i; magnetic conductivity /
    // permeability pairs when the structure has them
    const float *mh1y = EXT ? S.mag_h1[1] : nullptr, *mh2y = EXT ? S.mag_h2[1] : nullptr;
    // magnetic Lorentz poles: the curl updates B, H = B - sum M (tm_mpole4)
    const bool mp = MP && S.n_mpoles > 0;
    float hyP[4], hyN[4];
    {
        float byp[4];
        zero4(byp);
        if (mp && act && i >= 1) ld4(S.f_b[1][par] + ro - P, byp);
        tm_hy(S, i - 1, i >= 1, act, jb, hxbp, hxap, dt, rdx, ez0, ez1, mp ? byp : hyp, p1p,
              hyP, C.amp_h, mh1y, mh2y);
    }
    if (mp && act && i >= 1) tm_mpole4(S, C, 1, ro - P, false, hyp, hyP);
    if (i < 1) zero4(hyP);
    if (EXT && i == 0 && S.cut_x == 2 && act) {
        // odd x mirror / Rotate4: the on-plane Hy column is the ghost of row 0
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = jb + q;
            if (j < ny) {
                hyP[q] = tm_cut_line<EXPL, EXT>(S, C, 1, j, ez1[q], dt, rdx);
                S.f_y0[par ^ 1][j] = hyP[q];
            }
        }
    }
    {
        float byo[4];
        zero4(byo);
        if (mp && act) ld4(S.f_b[1][par] + ro, byo);
        tm_hy(S, i, hyRow, act, jb, hxb, hxa, dt, rdx, ez1, ez2, mp ? byo : hy, p1, hyN, C.amp_h,
              mh1y, mh2y);
    }
    if (mp && act) tm_mpole4(S, C, 1, ro, true, hy, hyN);

    // Hx(n+1/2) row i (core/stepper_tm.py:91-94, :121-128): Hx' = Hx - dt curl, or
    // h1x Hx - h2x curl with magnetic pairs (Bx with magnetic poles)
    const bool magx = EXT && S.mag_h1[0] != nullptr;
    float mx1[4] = {1.f, 1.f, 1.f, 1.f}, mx2[4] = {dt, dt, dt, dt};
    if (magx && act) {
        ld4(S.mag_h1[0] + ro, mx1);
        ld4(S.mag_h2[0] + ro, mx2);
    }
    float hxN[4], bxo[4];
    zero4(bxo);
    if (mp && act) ld4(S.f_b[0][par] + ro, bxo);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float er = (q < 3) ? ez1[q + 1] : ezR;
        const float d = (er - ez1[q]) * rdx;
        const float pv = hyb[q] * p0[q] + hya[q] * d;
        const float f = mp ? bxo[q] : hx[q];
        const float hn = magx ? mx1[q] * f - mx2[q] * (d + pv) : f - dt * (d + pv);
        hxN[q] = vH[q] ? hn : f;
        p0[q] = vH[q] ? pv : p0[q];
    }
    if (act && i >= S.src_h2.row_lo && i <= S.src_h2.row_hi) apply_cells(S.src_h2, i, C.amp_h, jb, hxN);
    if (mp && act) tm_mpole4(S, C, 0, ro, true, hx, hxN);
    // Hx(n+1/2)(i, jb-1): the left lane's last column; lane 0 recomputes its own
    float hxm0 = __shfl_up_sync(0xffffffffu, hxN[3], 1);
    if (lane == 0) {
        float v = 0.f;
        if (hasL) {
            const float d = (ez1[0] - ezl) * rdx;
            float c = d;
            if (byHL) c = d + (__ldg(S.hy_b + jl) * p0l + __ldg(S.hy_a + jl) * d);
            const float f = mp ? S.f_b[0][par][ro - 1] : hxl;
            v = magx ? S.mag_h1[0][ro - 1] * f - S.mag_h2[0][ro - 1] * c : f - dt * c;
            if (i >= S.src_h2.row_lo && i <= S.src_h2.row_hi)
                v = apply_cell1(S.src_h2, i, jl, C.amp_h, v);
            if (mp) v = tm_mpole1(S, C, 0, ro - 1, hxl, v);
        } else if (EXT && jb == 0 && S.cut_y == 2) {
            // odd y mirror / Rotate2 / Rotate4: the on-plane Hx row is the ghost of column 0
            v = tm_cut_line<EXPL, EXT>(S, C, 0, i, ez1[0], dt, rdx);
            S.f_x0[par ^ 1][i] = v;
        }
        hxm0 = v;
    }

    // Dz(n+1) row i (core/stepper_tm.py:136-166), electric source, Ez = Dz / eps;
    // with conductivity Dz' = c1 Dz + c2 curl, curl zero outside the updated cells
    const bool cond = EXT && S.cond_d1[0] != nullptr;
    float c1[4], c2[4];
    if (cond && act) {
        ld4(S.cond_d1[0] + ro, c1);
        ld4(S.cond_d2[0] + ro, c2);
    }
    float dzN[4], ezN[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float hxm = (q == 0) ? hxm0 : hxN[q - 1];
        const float dhy = (hyN[q] - hyP[q]) * rdx;
        const float dhx = (hxN[q] - hxm) * rdx;
        const float q2 = exb * p2[q] + exa * dhy;
        const float q3 = eyb[q] * p3[q] + eya[q] * dhx;
        const float curl = (dhy + q2) - (dhx + q3);
        const float dn = cond ? c1[q] * d1[q] + c2[q] * curl : d1[q] + dt * curl;
        dzN[q] = vD[q] ? dn : (cond ? c1[q] * d1[q] : d1[q]);
        p2[q] = vD[q] ? q2 : p2[q];
        p3[q] = vD[q] ? q3 : p3[q];
    }
    if (act && i >= S.src_e.row_lo && i <= S.src_e.row_hi) apply_cells(S.src_e, i, C.amp_e, jb, dzN);
    // ADE update P(n+1) = c1 P(n) + c2 P(n-1) + c3 Ez(n) into the third buffer
    // (core/stepper_tm.py:203-207), then Ez = (Dz - sum_k P_k) / eps
    float psN[4];
    zero4(psN);
    if (EXT && S.n_poles > 0 && act) {
        const float *Pc = S.pol_p[C.pst];
        const float *Pp = S.pol_p[(C.pst + 2) % 3];
        float *Po = S.pol_p[(C.pst + 1) % 3];
        const uint32_t pl = (uint32_t)nx * P;
#pragma unroll 1
        for (int k = 0; k < (EXT ? S.n_poles : 0); ++k) {
            const uint32_t o = k * pl + ro;
            float pc[4], pp[4], a1[4], a2[4], a3[4];
            ld4(Pc + o, pc);
            ld4(Pp + o, pp);
            ld4(S.pol_c[0] + o, a1);
            ld4(S.pol_c[1] + o, a2);
            ld4(S.pol_c[2] + o, a3);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                pc[q] = a1[q] * pc[q] + a2[q] * pp[q] + a3[q] * ez1[q];
                psN[q] += pc[q];
            }
            st4(Po + o, pc);
        }
    }
    {
        float rN[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) rN[q] = dzN[q] - psN[q];
        if (act) tm_e4(S, EXT && S.chi2 != nullptr, ro, rN, e1, ezN);
        else zero4(ezN);
    }
    if (!act) return;
    const int pn = par ^ 1;
    st4(S.f_main[pn] + ro, dzN);
    st4(S.f_x[pn] + ro, hxN);
    st4(S.f_y[pn] + ro, hyN);
    if (byH) st4(S.psi[0][pn] + ro, p0);
    if (bxH) st4(S.psi[1][pn] + ro, p1);
    if (bxE) st4(S.psi[2][pn] + ro, p2);
    if (byE) st4(S.psi[3][pn] + ro, p3);
    float *ring = C.ring;
    if (S.ring_full[0] >= 0) st4(ring + S.ring_full[0] + ro, ezN);
    if (S.ring_full[1] >= 0) st4(ring + S.ring_full[1] + ro, hxN);
    if (S.ring_full[2] >= 0) st4(ring + S.ring_full[2] + ro, hyN);
    if (nl) {
        sample_row(L, nl, MTB_C2_MAIN, i, jb, true, ezN, ring);
        sample_row(L, nl, MTB_C2_X, i, jb, true, hxN, ring);
        sample_row(L, nl, MTB_C2_Y, i, jb, true, hyN, ring);
    }
}

// Dy(n+1/2) of one row from Hz rows r-1 (hp), r (hc): core/stepper_te.py:79-111,
// source :120-134. `valid` = 1 <= r <= nx-2.
// Sum over a pole stack (planes pl floats apart) of one float4 at offset o.
__device__ __forceinline__ void pole_sum4(const float *Pc, int np, uint32_t pl, uint32_t o,
                                          float (&s)[4]) {
    zero4(s);
#pragma unroll 1
    for (int k = 0; k < np; ++k) {
        float t[4];
        ld4(Pc + k * pl + o, t);
#pragma unroll
        for (int q = 0; q < 4; ++q) s[q] += t[q];
    }
}

// ADE step of one float4 of a pole stack: P(n+1) = c1 P(n) + c2 P(n-1) + c3 E(n)
// (core/stepper_tm.py:203-207, core/stepper_te.py:136-146), written to the third
// buffer when STORE (the owner of the cells), and sum_k P_k(n+1) into s.
template <bool STORE>
__device__ __forceinline__ void pole_step4(const float *Pc, const float *Pp, float *Po,
                                           const float *const *c, int np, uint32_t pl,
                                           uint32_t o, const float (&e)[4], float (&s)[4]) {
    zero4(s);
#pragma unroll 1
    for (int k = 0; k < np; ++k) {
        const uint32_t ok = k * pl + o;
        float pc[4], pp[4], a1[4], a2[4], a3[4];
        ld4(Pc + ok, pc);
        ld4(Pp + ok, pp);
        ld4(c[0] + ok, a1);
        ld4(c[1] + ok, a2);
        ld4(c[2] + ok, a3);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            pc[q] = a1[q] * pc[q] + a2[q] * pp[q] + a3[q] * e[q];
            s[q] += pc[q];
        }
        if (STORE) st4(Po + ok, pc);
    }
}

template <bool EXT>
__device__ __forceinline__ void te_dy(const mtb_yee2d_struct &S, int r, bool valid, bool act,
                                      int jb, float b, float a, float dt, float rdx,
                                      const float (&hp)[4], const float (&hc)[4],
                                      const float (&dy)[4], float (&ps)[4], float (&out)[4],
                                      const float *amp_e) {
    // conductivity: Dy' = c1 Dy - c2 curl, curl zero outside the updated cells
    // (core/stepper_te.py D update with d1y / d2y); rows past the grid keep Dy
    const bool cond = EXT && S.cond_d1[1] != nullptr;
    float c1[4], c2[4];
    if (cond && act && r < S.nx) {
        const uint32_t o = (uint32_t)r * S.pitch + jb;
        ld4(S.cond_d1[1] + o, c1);
        ld4(S.cond_d2[1] + o, c2);
    } else {
        c1[0] = c1[1] = c1[2] = c1[3] = 1.f;
        zero4(c2);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const bool v = valid && act && jb + q <= S.ny - 2;
        const float d = (hc[q] - hp[q]) * rdx;
        const float pv = b * ps[q] + a * d;
        const float dn = cond ? c1[q] * dy[q] - c2[q] * (d + pv) : dy[q] - dt * (d + pv);
        out[q] = v ? dn : (cond ? c1[q] * dy[q] : dy[q]);
        ps[q] = v ? pv : ps[q];
    }
    if (act && r >= S.src_e.row_lo && r <= S.src_e.row_hi) apply_cells(S.src_e, r, amp_e, jb, out);
}

template <bool EXT>
__device__ __forceinline__ void te_tile(const mtb_yee2d_struct &S, const int i, const int c0,
                                        const Ctx2D &C, const mtb_line_sample *L, const int nl) {
    const int lane = threadIdx.x;
    const int nx = S.nx, ny = S.ny, P = S.pitch;
    const int jb = c0 + 4 * lane;
    const bool act = jb < P;
    const float dt = S.dt, rdx = 1.0f / S.dx;
    const int par = C.par;
    const uint32_t ro = (uint32_t)i * P + jb;
    const float *__restrict__ Hz = S.f_main[par];
    const float *__restrict__ Dx = S.f_x[par];
    const float *__restrict__ Dy = S.f_y[par];
    const float *__restrict__ iex = S.inv_eps_a;
    const float *__restrict__ iey = S.inv_eps_b;
    // even symmetry cuts (core/stepper_te.py:88-97): the cut row of Dy (x cut) and
    // column of Dx (y cut) are live with dHz/dn = 2 Hz / dx (odd Hz ghost)
    const bool cutx = EXT && S.cut_x != 0, cuty = EXT && S.cut_y != 0;
    const bool hzRow = i <= nx - 2;                     // Hz, Dx (Ex) rows
    const bool dyRow = (i >= 1 || cutx) && i <= nx - 2, dyRowN = i + 1 <= nx - 2;
    const bool bxH = hzRow && in_band(i, S.xband[0], S.xband[1]);
    const bool bxE = dyRow && in_band(i, S.xband[2], S.xband[3]);
    const bool bxEn = dyRowN && in_band(i + 1, S.xband[2], S.xband[3]);
    const bool byE = act && hzRow && band4(jb, S.yband[2], S.yband[3]);
    const bool byH = act && hzRow && band4(jb, S.yband[0], S.yband[1]);
    const int jr = jb + 4;
    const bool hasR = lane == 31 && hzRow && jr <= ny - 1;
    const bool updR = hasR && jr >= 1 && jr <= ny - 2;
    const bool byER = updR && in_band(jr, S.yband[2], S.yband[3]);

    float hc[4], hp[4], hn[4], dx[4], dy[4], dyn[4], ix[4], iy[4], iyn[4];
    float p0[4], p1[4], p1n[4], p2[4], p3[4];
    float hzL = 0.f, hzR = 0.f, dxr = 0.f, ixr = 0.f, p0r = 0.f;
    zero4(hc); zero4(hp); zero4(hn); zero4(dx); zero4(dy); zero4(dyn); zero4(ix); zero4(iy);
    zero4(iyn); zero4(p0); zero4(p1); zero4(p1n); zero4(p2); zero4(p3);
    if (act) {
        ld4(Hz + ro, hc);
        ld4(Dx + ro, dx);
        ld4(Dy + ro, dy);
        ld4(iex + ro, ix);
        ld4(iey + ro, iy);
        if (i >= 1) ld4(Hz + ro - P, hp);
        if (i + 1 < nx) { ld4(Hz + ro + P, hn); ld4(Dy + ro + P, dyn); ld4(iey + ro + P, iyn); }
        if (lane == 0 && jb >= 1) hzL = Hz[ro - 1];
        if (hasR) {
            hzR = Hz[ro + 4];
            dxr = Dx[ro + 4];
            ixr = iex[ro + 4];
            if (byER) p0r = S.psi[0][par][ro + 4];
        }
        if (byE) ld4(S.psi[0][par] + ro, p0);
        if (bxE) ld4(S.psi[1][par] + ro, p1);
        if (bxEn) ld4(S.psi[1][par] + ro + P, p1n);
        if (bxH) ld4(S.psi[2][par] + ro, p2);
        if (byH) ld4(S.psi[3][par] + ro, p3);
    }
    float hxb = 1.f, hxa = 0.f, exb = 1.f, exa = 0.f, exbn = 1.f, exan = 0.f;
    if (bxH) { hxb = __ldg(S.hx_b + i); hxa = __ldg(S.hx_a + i); }
    if (bxE) { exb = __ldg(S.ex_b + i); exa = __ldg(S.ex_a + i); }
    if (bxEn) { exbn = __ldg(S.ex_b + i + 1); exan = __ldg(S.ex_a + i + 1); }
    float hyb[4], hya[4], eyb[4], eya[4];
    bool vX[4], vZ[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        vX[q] = act && hzRow && (j >= 1 || cuty) && j <= ny - 2;
        vZ[q] = act && hzRow && j <= ny - 2;
        const bool oe = byE && j >= 1 && j <= ny - 2, oh = byH && j <= ny - 2;
        eyb[q] = oe ? __ldg(S.ey_b + j) : 1.f;
        eya[q] = oe ? __ldg(S.ey_a + j) : 0.f;
        hyb[q] = oh ? __ldg(S.hy_b + j) : 1.f;
        hya[q] = oh ? __ldg(S.hy_a + j) : 0.f;
    }
    float hm0 = __shfl_up_sync(0xffffffffu, hc[3], 1);
    if (lane == 0) hm0 = (cuty && jb == 0) ? -hc[0] : hzL;

    // Dx / Ex(n+1/2) row i (core/stepper_te.py:79-95, :150-160)
    float dxN[4], ex[4];
    // conductivity: Dx' = c1 Dx + c2 curl (core/stepper_te.py D update, d1x / d2x)
    const bool cond = EXT && S.cond_d1[0] != nullptr;
    float c1[4], c2[4];
    if (cond && act) {
        ld4(S.cond_d1[0] + ro, c1);
        ld4(S.cond_d2[0] + ro, c2);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float hm = (q == 0) ? hm0 : hc[q - 1];
        const float d = (hc[q] - hm) * rdx;
        const float pv = eyb[q] * p0[q] + eya[q] * d;
        const float dn = cond ? c1[q] * dx[q] + c2[q] * (d + pv) : dx[q] + dt * (d + pv);
        dxN[q] = vX[q] ? dn : (cond ? c1[q] * dx[q] : dx[q]);
        p0[q] = vX[q] ? pv : p0[q];
        ex[q] = hzRow ? dxN[q] * ix[q] : 0.f;
    }
    // dispersive poles on Ex / Ey (core/stepper_te.py:136-175): the ADE step on
    // the old E, then E = (D - sum P) / eps; the halo cells (lane 31's column,
    // row i+1 of Ey) recompute their poles without storing them
    const int npx = EXT ? S.n_poles : 0, npy = EXT ? S.n_poles_y : 0;
    const uint32_t pl = (uint32_t)nx * P;
    if (npx > 0 && act) {
        float sc[4], eo[4], sn[4];
        pole_sum4(S.pol_p[C.pst], npx, pl, ro, sc);
#pragma unroll
        for (int q = 0; q < 4; ++q) eo[q] = (dx[q] - sc[q]) * ix[q];
        pole_step4<true>(S.pol_p[C.pst], S.pol_p[(C.pst + 2) % 3], S.pol_p[(C.pst + 1) % 3],
                         S.pol_c, npx, pl, ro, eo, sn);
#pragma unroll
        for (int q = 0; q < 4; ++q) ex[q] = hzRow ? (dxN[q] - sn[q]) * ix[q] : 0.f;
    }
    // Ex(n+1/2)(i, jb+4): lane 31's right neighbour column
    float exR = 0.f;
    if (hasR) {
        float v = dxr;
        const float c1r = cond ? S.cond_d1[0][ro + 4] : 1.f;
        if (updR) {
            const float d = (hzR - hc[3]) * rdx;
            float c = d;
            if (byER) c = d + (__ldg(S.ey_b + jr) * p0r + __ldg(S.ey_a + jr) * d);
            v = cond ? c1r * dxr + S.cond_d2[0][ro + 4] * c : dxr + dt * c;
        } else if (cond) {
            v = c1r * dxr;
        }
        float sN = 0.f;
        if (npx > 0) {
            const float *Pc = S.pol_p[C.pst], *Pp = S.pol_p[(C.pst + 2) % 3];
            float sc = 0.f;
            for (int k = 0; k < npx; ++k) sc += Pc[k * pl + ro + 4];
            const float eo = (dxr - sc) * ixr;
            for (int k = 0; k < npx; ++k) {
                const uint32_t ok = k * pl + ro + 4;
                sN += S.pol_c[0][ok] * Pc[ok] + S.pol_c[1][ok] * Pp[ok] + S.pol_c[2][ok] * eo;
            }
        }
        exR = (v - sN) * ixr;
    }
    // Dy / Ey(n+1/2) rows i and i+1 (recomputed halo)
    float dyN[4], ey[4], dyNn[4], eyn[4];
    if (cutx && i == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) hp[q] = -hc[q];
    }
    te_dy<EXT>(S, i, dyRow, act, jb, exb, exa, dt, rdx, hp, hc, dy, p1, dyN, C.amp_e);
    te_dy<EXT>(S, i + 1, dyRowN, act, jb, exbn, exan, dt, rdx, hc, hn, dyn, p1n, dyNn, C.amp_e);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        ey[q] = dyN[q] * iy[q];
        eyn[q] = (i + 1 < nx) ? dyNn[q] * iyn[q] : 0.f;
    }
    if (npy > 0 && act) {
        float sc[4], eo[4], sn[4];
        const float *Pc = S.pol_py[C.pst], *Pp = S.pol_py[(C.pst + 2) % 3];
        float *Po = S.pol_py[(C.pst + 1) % 3];
        pole_sum4(Pc, npy, pl, ro, sc);
#pragma unroll
        for (int q = 0; q < 4; ++q) eo[q] = (dy[q] - sc[q]) * iy[q];
        pole_step4<true>(Pc, Pp, Po, S.pol_cy, npy, pl, ro, eo, sn);
#pragma unroll
        for (int q = 0; q < 4; ++q) ey[q] = (dyN[q] - sn[q]) * iy[q];
        if (i + 1 < nx) {
            pole_sum4(Pc, npy, pl, ro + P, sc);
#pragma unroll
            for (int q = 0; q < 4; ++q) eo[q] = (dyn[q] - sc[q]) * iyn[q];
            pole_step4<false>(Pc, Pp, Po, S.pol_cy, npy, pl, ro + P, eo, sn);
#pragma unroll
            for (int q = 0; q < 4; ++q) eyn[q] = (dyNn[q] - sn[q]) * iyn[q];
        }
    }
    float exr = __shfl_down_sync(0xffffffffu, ex[0], 1);
    if (lane == 31) exr = exR;

    // Hz(n+1) row i (core/stepper_te.py:113-117): Hz' = Hz - dt curl, or
    // hz1 Hz - hz2 curl with magnetic conductivity / permeability
    const bool magz = EXT && S.mag_h1[0] != nullptr;
    float mz1[4] = {1.f, 1.f, 1.f, 1.f}, mz2[4] = {dt, dt, dt, dt};
    if (magz && act) {
        ld4(S.mag_h1[0] + ro, mz1);
        ld4(S.mag_h2[0] + ro, mz2);
    }
    float hzN[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float exn = (q < 3) ? ex[q + 1] : exr;
        const float dey = (eyn[q] - ey[q]) * rdx;
        const float dex = (exn - ex[q]) * rdx;
        const float q2 = hxb * p2[q] + hxa * dey;
        const float q3 = hyb[q] * p3[q] + hya[q] * dex;
        const float cz = (dey + q2) - (dex + q3);
        const float hn_ = magz ? mz1[q] * hc[q] - mz2[q] * cz : hc[q] - dt * cz;
        hzN[q] = vZ[q] ? hn_ : hc[q];
        p2[q] = vZ[q] ? q2 : p2[q];
        p3[q] = vZ[q] ? q3 : p3[q];
    }
    if (act && hzRow && i >= S.src_h1.row_lo && i <= S.src_h1.row_hi)
        apply_cells(S.src_h1, i, C.amp_h, jb, hzN);
    if (!act) return;
    const int pn = par ^ 1;
    st4(S.f_main[pn] + ro, hzN);
    st4(S.f_x[pn] + ro, dxN);
    st4(S.f_y[pn] + ro, dyN);
    if (byE) st4(S.psi[0][pn] + ro, p0);
    if (bxE) st4(S.psi[1][pn] + ro, p1);
    if (bxH) st4(S.psi[2][pn] + ro, p2);
    if (byH) st4(S.psi[3][pn] + ro, p3);
    float *ring = C.ring;
    if (S.ring_full[0] >= 0) st4(ring + S.ring_full[0] + ro, hzN);
    if (S.ring_full[1] >= 0) st4(ring + S.ring_full[1] + ro, ex);
    if (S.ring_full[2] >= 0) st4(ring + S.ring_full[2] + ro, ey);
    if (nl) {
        sample_row(L, nl, MTB_C2_MAIN, i, jb, true, hzN, ring);
        sample_row(L, nl, MTB_C2_X, i, jb, true, ex, ring);
        sample_row(L, nl, MTB_C2_Y, i, jb, true, ey, ring);
    }
}

// Lean TM rows: rows ib .. ib+R-1 of one warp, all in [1, nx-2] and outside
// the x layers (no x-direction CPML memory), columns jb .. jb+3 of one lane.
// The R rows share their neighbour rows' loads (R+2 rows of Dz and 1/eps,
// R+1 of Hy): per cell a fraction of tm_tile's loads and index work. YPSI adds
// the y-direction CPML of lanes inside a y layer. Same arithmetic as tm_tile
// (the x-CPML terms there are b psi + a d = 0 here), so either path may
// recompute a neighbour's halo row.
template <int R, bool YPSI>
__device__ __forceinline__ void tm_rows(const mtb_yee2d_struct &S, const int ib, const int c0,
                                        const Ctx2D &C, const mtb_line_sample *L, const int nl) {
    const int lane = threadIdx.x;
    const int ny = S.ny, P = S.pitch;
    const int jb = c0 + 4 * lane;
    const bool act = jb < P;
    const float dt = S.dt, rdx = 1.0f / S.dx;
    const int par = C.par;
    const float *__restrict__ Dz = S.f_main[par];
    const float *__restrict__ Hx = S.f_x[par];
    const float *__restrict__ Hy = S.f_y[par];
    const float *__restrict__ ie = S.inv_eps_a;
    // lanes past the row end (last strip) read the row's last float4 instead:
    // their results are never stored and feed only masked neighbour cells
    const uint32_t o0 = (uint32_t)ib * P + (act ? jb : P - 4);   // own row 0
    const uint32_t om = o0 - P;                         // row ib-1 (ib >= 1)
    const int jl = jb - 1;
    const bool hasL = lane == 0 && jl >= 0 && jl <= ny - 2;
    const bool byH = YPSI && act && band4(jb, S.yband[0], S.yband[1]);
    const bool byE = YPSI && act && band4(jb, S.yband[2], S.yband[3]);
    const bool byHL = YPSI && hasL && in_band(jl, S.yband[0], S.yband[1]);
    const bool rok = lane == 31 && jb + 4 < P;

    float dv[R + 2][4], iv[R + 2][4];                  // Dz, 1/eps rows ib-1 .. ib+R
    float hx[R][4], hy[R + 1][4];                      // Hx own rows; Hy rows ib-1 .. ib+R-1
    float ezl[R], ezr[R], hxl[R], p0l[R];
    float p0[R][4], p3[R][4];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        zero4(p0[r]); zero4(p3[r]);
        ezl[r] = ezr[r] = hxl[r] = p0l[r] = 0.f;
    }
#pragma unroll
    for (int k = 0; k < R + 2; ++k) {
        ld4(Dz + om + k * P, dv[k]);
        ld4(ie + om + k * P, iv[k]);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) ld4(Hx + o0 + r * P, hx[r]);
#pragma unroll
    for (int k = 0; k < R + 1; ++k) ld4(Hy + om + k * P, hy[k]);
    if (act) {
        if (lane == 0 && jl >= 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                ezl[r] = Dz[o0 + r * P - 1] * ie[o0 + r * P - 1];
                if (hasL) hxl[r] = Hx[o0 + r * P - 1];
                if (byHL) p0l[r] = S.psi[0][par][o0 + r * P - 1];
            }
        }
        if (rok) {
#pragma unroll
            for (int r = 0; r < R; ++r) ezr[r] = Dz[o0 + r * P + 4] * ie[o0 + r * P + 4];
        }
        if (YPSI) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (byH) ld4(S.psi[0][par] + o0 + r * P, p0[r]);
                if (byE) ld4(S.psi[3][par] + o0 + r * P, p3[r]);
            }
        }
    }
    const bool pmc = S.y_pmc != 0;
    float hyb[4], hya[4], eyb[4], eya[4];
    bool vH[4], vD[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        vH[q] = act && j <= ny - 2;
        vD[q] = act && (pmc ? (j < ny) : (j >= 1 && j <= ny - 2));
        hyb[q] = 1.f; hya[q] = 0.f; eyb[q] = 1.f; eya[q] = 0.f;
        if (YPSI) {
            const bool oh = byH && j <= ny - 2, oe = byE && j < ny;
            if (oh) { hyb[q] = __ldg(S.hy_b + j); hya[q] = __ldg(S.hy_a + j); }
            if (oe) { eyb[q] = __ldg(S.ey_b + j); eya[q] = __ldg(S.ey_a + j); }
        }
    }
    float ez[R + 2][4];
#pragma unroll
    for (int k = 0; k < R + 2; ++k)
#pragma unroll
        for (int q = 0; q < 4; ++q) ez[k][q] = dv[k][q] * iv[k][q];

    // Hy(n+1/2) rows ib-1 .. ib+R-1 (all <= nx-2, outside the x layers)
    float hyN[R + 1][4];
#pragma unroll
    for (int k = 0; k < R + 1; ++k) {
        const int row = ib - 1 + k;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            hyN[k][q] = hy[k][q] + dt * ((ez[k + 1][q] - ez[k][q]) * rdx);
        }
        if (act && row >= S.src_h1.row_lo && row <= S.src_h1.row_hi)
            apply_cells(S.src_h1, row, C.amp_h, jb, hyN[k]);
    }
    float *ring = C.ring;
    const int pn = par ^ 1;
    // descriptor fields used after the first global store, held in registers
    // (the stores could alias the shared descriptor, which would force reloads)
    const int h2_lo = S.src_h2.row_lo, h2_hi = S.src_h2.row_hi;
    const int e_lo = S.src_e.row_lo, e_hi = S.src_e.row_hi;
    float *__restrict__ dzo = S.f_main[pn];
    float *__restrict__ hxo = S.f_x[pn];
    float *__restrict__ hyo = S.f_y[pn];
    float *__restrict__ ps0o = S.psi[0][pn];
    float *__restrict__ ps3o = S.psi[3][pn];
    float *__restrict__ rE = S.ring_full[0] >= 0 ? ring + S.ring_full[0] : nullptr;
    float *__restrict__ rX = S.ring_full[1] >= 0 ? ring + S.ring_full[1] : nullptr;
    float *__restrict__ rY = S.ring_full[2] >= 0 ? ring + S.ring_full[2] : nullptr;
    float hylb = 0.f, hyla = 0.f;
    if (YPSI && byHL) { hylb = __ldg(S.hy_b + jl); hyla = __ldg(S.hy_a + jl); }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = ib + r;
        const uint32_t ro = o0 + r * P;
        // Hx(n+1/2) row i
        float ezR = __shfl_down_sync(0xffffffffu, ez[r + 1][0], 1);
        if (lane == 31) ezR = ezr[r];
        float hxN[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float er = (q < 3) ? ez[r + 1][q + 1] : ezR;
            const float d = (er - ez[r + 1][q]) * rdx;
            float hn;
            if (YPSI) {
                const float pv = hyb[q] * p0[r][q] + hya[q] * d;
                hn = hx[r][q] - dt * (d + pv);
                p0[r][q] = vH[q] ? pv : p0[r][q];
            } else {
                hn = hx[r][q] - dt * d;
            }
            hxN[q] = vH[q] ? hn : hx[r][q];
        }
        if (act && i >= h2_lo && i <= h2_hi) apply_cells(S.src_h2, i, C.amp_h, jb, hxN);
        float hxm0 = __shfl_up_sync(0xffffffffu, hxN[3], 1);
        if (lane == 0) {
            float v = 0.f;
            if (hasL) {
                const float d = (ez[r + 1][0] - ezl[r]) * rdx;
                float c = d;
                if (byHL) c = d + (hylb * p0l[r] + hyla * d);
                v = hxl[r] - dt * c;
                if (i >= h2_lo && i <= h2_hi) v = apply_cell1(S.src_h2, i, jl, C.amp_h, v);
            }
            hxm0 = v;
        }
        // Dz(n+1) row i, electric source, Ez = Dz / eps
        float dzN[4], ezN[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float hxm = (q == 0) ? hxm0 : hxN[q - 1];
            const float dhy = (hyN[r + 1][q] - hyN[r][q]) * rdx;
            const float dhx = (hxN[q] - hxm) * rdx;
            float dn;
            if (YPSI) {
                const float q3 = eyb[q] * p3[r][q] + eya[q] * dhx;
                dn = dv[r + 1][q] + dt * (dhy - (dhx + q3));
                p3[r][q] = vD[q] ? q3 : p3[r][q];
            } else {
                dn = dv[r + 1][q] + dt * (dhy - dhx);
            }
            dzN[q] = vD[q] ? dn : dv[r + 1][q];
        }
        if (act && i >= e_lo && i <= e_hi) apply_cells(S.src_e, i, C.amp_e, jb, dzN);
#pragma unroll
        for (int q = 0; q < 4; ++q) ezN[q] = dzN[q] * iv[r + 1][q];
        if (act) {
            st4(dzo + ro, dzN);
            st4(hxo + ro, hxN);
            st4(hyo + ro, hyN[r + 1]);
            if (YPSI && byH) st4(ps0o + ro, p0[r]);
            if (YPSI && byE) st4(ps3o + ro, p3[r]);
            if (rE) st4(rE + ro, ezN);
            if (rX) st4(rX + ro, hxN);
            if (rY) st4(rY + ro, hyN[r + 1]);
            if (nl) {
                sample_row(L, nl, MTB_C2_MAIN, i, jb, true, ezN, ring);
                sample_row(L, nl, MTB_C2_X, i, jb, true, hxN, ring);
                sample_row(L, nl, MTB_C2_Y, i, jb, true, hyN[r + 1], ring);
            }
        }
    }
}

template <bool FIRST, bool EXT, bool MP = false>
__global__ void __launch_bounds__(32 * TROWS, 2) k_tile_tm(
    const mtb_yee2d_struct *__restrict__ SS, const int4 *__restrict__ work, int n_work,
    Ctx2D C) {
    __shared__ TileSmem T;
    int4 w;
    if (!tile_setup(SS, work, n_work, C.wr, T, w)) return;
    const mtb_yee2d_struct &S = T.s;
    const int ib = w.y + threadIdx.y * C.wr;           // this warp's rows ib .. ib+wr-1
    if (ib >= S.nx) return;                             // whole warp
    const bool expl = FIRST && S.explicit_e;
    // lean rows: interior rows outside the x layers, imported Ez not pending
    const int last = ib + WROWS - 1;
    const bool lean = C.wr == WROWS && !expl && ib >= 1 && last <= S.nx - 2 &&
                      ib - 1 >= S.xband[0] && last < S.xband[1] &&
                      ib >= S.xband[2] && last < S.xband[3] && S.cond_d1[0] == nullptr &&
                      S.n_poles == 0 && S.mag_h1[0] == nullptr && S.mag_h1[1] == nullptr &&
                      S.chi2 == nullptr && S.n_mpoles == 0 && !(EXT && S.cut_y && w.z == 0);
    if (lean) {
        const int jb = w.z + 4 * threadIdx.x;
        const bool yb = jb < S.pitch &&
                        (band4(jb, S.yband[0], S.yband[1]) || band4(jb, S.yband[2], S.yband[3]) ||
                         (threadIdx.x == 0 && jb >= 1 && in_band(jb - 1, S.yband[0], S.yband[1])));
        if (!__any_sync(0xffffffffu, yb)) {
            tm_rows<WROWS, false>(S, ib, w.z, C, T.lines, T.nl);
        } else {
#pragma unroll 1
            for (int h = 0; h < WROWS; h += 2) tm_rows<2, true>(S, ib + h, w.z, C, T.lines, T.nl);
        }
        return;
    }
#pragma unroll 1
    for (int r = 0; r < C.wr; ++r) {
        if (ib + r >= S.nx) break;
        if (FIRST && expl)
            tm_tile<true, EXT, MP>(S, ib + r, w.z, C, T.lines, T.nl);
        else
            tm_tile<false, EXT, MP>(S, ib + r, w.z, C, T.lines, T.nl);
    }
}

// Lean TE rows: Hz rows ib .. ib+R-1 of one warp with their Dx / Ex rows and
// the Dy / Ey rows ib .. ib+R (the last one is the halo the Hz update needs),
// all in [1, nx-2] and outside the x layers; y-direction CPML when YPSI. Same
// arithmetic as te_tile / te_dy.
template <int R, bool YPSI>
__device__ __forceinline__ void te_rows(const mtb_yee2d_struct &S, const int ib, const int c0,
                                        const Ctx2D &C, const mtb_line_sample *L, const int nl) {
    const int lane = threadIdx.x;
    const int ny = S.ny, P = S.pitch;
    const int jb = c0 + 4 * lane;
    const bool act = jb < P;
    const float dt = S.dt, rdx = 1.0f / S.dx;
    const int par = C.par;
    const float *__restrict__ Hz = S.f_main[par];
    const float *__restrict__ Dx = S.f_x[par];
    const float *__restrict__ Dy = S.f_y[par];
    const float *__restrict__ iex = S.inv_eps_a;
    const float *__restrict__ iey = S.inv_eps_b;
    // lanes past the row end (last strip) read the row's last float4 instead:
    // their results are never stored and feed only masked neighbour cells
    const uint32_t o0 = (uint32_t)ib * P + (act ? jb : P - 4);
    const uint32_t om = o0 - P;                         // row ib-1 (ib >= 1)
    const int jr = jb + 4;
    const bool hasR = lane == 31 && jr <= ny - 1;
    const bool updR = hasR && jr <= ny - 2;             // jr >= 1 always
    const bool byE = YPSI && act && band4(jb, S.yband[2], S.yband[3]);
    const bool byH = YPSI && act && band4(jb, S.yband[0], S.yband[1]);
    const bool byER = YPSI && updR && in_band(jr, S.yband[2], S.yband[3]);

    float hz[R + 2][4];                                 // Hz rows ib-1 .. ib+R
    float dx[R][4], ix[R][4];                           // Dx, 1/eps_x own rows
    float dy[R + 1][4], iy[R + 1][4];                   // Dy, 1/eps_y rows ib .. ib+R
    float hzL[R], hzR[R], dxr[R], ixr[R], p0r[R];
    float p0[R][4], p3[R][4];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        zero4(p0[r]); zero4(p3[r]);
        hzL[r] = hzR[r] = dxr[r] = ixr[r] = p0r[r] = 0.f;
    }
#pragma unroll
    for (int k = 0; k < R + 2; ++k) ld4(Hz + om + k * P, hz[k]);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        ld4(Dx + o0 + r * P, dx[r]);
        ld4(iex + o0 + r * P, ix[r]);
    }
#pragma unroll
    for (int k = 0; k < R + 1; ++k) {
        ld4(Dy + o0 + k * P, dy[k]);
        ld4(iey + o0 + k * P, iy[k]);
    }
    if (act) {
        if (lane == 0 && jb >= 1) {
#pragma unroll
            for (int r = 0; r < R; ++r) hzL[r] = Hz[o0 + r * P - 1];
        }
        if (hasR) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                hzR[r] = Hz[o0 + r * P + 4];
                dxr[r] = Dx[o0 + r * P + 4];
                ixr[r] = iex[o0 + r * P + 4];
                if (byER) p0r[r] = S.psi[0][par][o0 + r * P + 4];
            }
        }
        if (YPSI) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (byE) ld4(S.psi[0][par] + o0 + r * P, p0[r]);
                if (byH) ld4(S.psi[3][par] + o0 + r * P, p3[r]);
            }
        }
    }
    float hyb[4], hya[4], eyb[4], eya[4];
    bool vX[4], vZ[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        vX[q] = act && j >= 1 && j <= ny - 2;
        vZ[q] = act && j <= ny - 2;
        hyb[q] = 1.f; hya[q] = 0.f; eyb[q] = 1.f; eya[q] = 0.f;
        if (YPSI) {
            const bool oe = byE && j >= 1 && j <= ny - 2, oh = byH && j <= ny - 2;
            if (oe) { eyb[q] = __ldg(S.ey_b + j); eya[q] = __ldg(S.ey_a + j); }
            if (oh) { hyb[q] = __ldg(S.hy_b + j); hya[q] = __ldg(S.hy_a + j); }
        }
    }
    // Dy / Ey(n+1/2) rows ib .. ib+R (te_dy outside the x layers)
    float ey[R + 1][4], dyN[R + 1][4];
#pragma unroll
    for (int k = 0; k < R + 1; ++k) {
        const int row = ib + k;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float dn = dy[k][q] - dt * ((hz[k + 1][q] - hz[k][q]) * rdx);
            dyN[k][q] = vZ[q] ? dn : dy[k][q];
        }
        if (act && row >= S.src_e.row_lo && row <= S.src_e.row_hi)
            apply_cells(S.src_e, row, C.amp_e, jb, dyN[k]);
#pragma unroll
        for (int q = 0; q < 4; ++q) ey[k][q] = dyN[k][q] * iy[k][q];
    }
    float *ring = C.ring;
    const int pn = par ^ 1;
    // descriptor fields used after the first global store, held in registers
    // (the stores could alias the shared descriptor, which would force reloads)
    const int h1_lo = S.src_h1.row_lo, h1_hi = S.src_h1.row_hi;
    float *__restrict__ hzo = S.f_main[pn];
    float *__restrict__ dxo = S.f_x[pn];
    float *__restrict__ dyo = S.f_y[pn];
    float *__restrict__ ps0o = S.psi[0][pn];
    float *__restrict__ ps3o = S.psi[3][pn];
    float *__restrict__ rZ = S.ring_full[0] >= 0 ? ring + S.ring_full[0] : nullptr;
    float *__restrict__ rX = S.ring_full[1] >= 0 ? ring + S.ring_full[1] : nullptr;
    float *__restrict__ rY = S.ring_full[2] >= 0 ? ring + S.ring_full[2] : nullptr;
    float eyrb = 0.f, eyra = 0.f;
    if (YPSI && byER) { eyrb = __ldg(S.ey_b + jr); eyra = __ldg(S.ey_a + jr); }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = ib + r;
        const uint32_t ro = o0 + r * P;
        const float (&hc)[4] = hz[r + 1];
        // Dx / Ex(n+1/2) row i
        float hm0 = __shfl_up_sync(0xffffffffu, hc[3], 1);
        if (lane == 0) hm0 = hzL[r];
        float dxN[4], ex[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float hm = (q == 0) ? hm0 : hc[q - 1];
            const float d = (hc[q] - hm) * rdx;
            float dn;
            if (YPSI) {
                const float pv = eyb[q] * p0[r][q] + eya[q] * d;
                dn = dx[r][q] + dt * (d + pv);
                p0[r][q] = vX[q] ? pv : p0[r][q];
            } else {
                dn = dx[r][q] + dt * d;
            }
            dxN[q] = vX[q] ? dn : dx[r][q];
            ex[q] = dxN[q] * ix[r][q];
        }
        float exR = 0.f;
        if (hasR) {
            float v = dxr[r];
            if (updR) {
                const float d = (hzR[r] - hc[3]) * rdx;
                float c = d;
                if (byER) c = d + (eyrb * p0r[r] + eyra * d);
                v = dxr[r] + dt * c;
            }
            exR = v * ixr[r];
        }
        float exr = __shfl_down_sync(0xffffffffu, ex[0], 1);
        if (lane == 31) exr = exR;
        // Hz(n+1) row i
        float hzN[4];
        const float (&eyo)[4] = ey[r];
        const float (&eyn)[4] = ey[r + 1];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float exn = (q < 3) ? ex[q + 1] : exr;
            const float dey = (eyn[q] - eyo[q]) * rdx;
            const float dex = (exn - ex[q]) * rdx;
            float hn;
            if (YPSI) {
                const float q3 = hyb[q] * p3[r][q] + hya[q] * dex;
                hn = hc[q] - dt * (dey - (dex + q3));
                p3[r][q] = vZ[q] ? q3 : p3[r][q];
            } else {
                hn = hc[q] - dt * (dey - dex);
            }
            hzN[q] = vZ[q] ? hn : hc[q];
        }
        if (act && i >= h1_lo && i <= h1_hi) apply_cells(S.src_h1, i, C.amp_h, jb, hzN);
        if (act) {
            st4(hzo + ro, hzN);
            st4(dxo + ro, dxN);
            st4(dyo + ro, dyN[r]);
            if (YPSI && byE) st4(ps0o + ro, p0[r]);
            if (YPSI && byH) st4(ps3o + ro, p3[r]);
            if (rZ) st4(rZ + ro, hzN);
            if (rX) st4(rX + ro, ex);
            if (rY) st4(rY + ro, eyo);
            if (nl) {
                sample_row(L, nl, MTB_C2_MAIN, i, jb, true, hzN, ring);
                sample_row(L, nl, MTB_C2_X, i, jb, true, ex, ring);
                sample_row(L, nl, MTB_C2_Y, i, jb, true, eyo, ring);
            }
        }
    }
}

template <bool EXT>
__global__ void __launch_bounds__(32 * TROWS, 2) k_tile_te(
    const mtb_yee2d_struct *__restrict__ SS, const int4 *__restrict__ work, int n_work,
    Ctx2D C) {
    __shared__ TileSmem T;
    int4 w;
    if (!tile_setup(SS, work, n_work, C.wr, T, w)) return;
    const mtb_yee2d_struct &S = T.s;
    const int ib = w.y + threadIdx.y * C.wr;
    if (ib >= S.nx) return;
    const int last = ib + WROWS - 1;
    // lean rows: Dy rows ib .. last+1 interior, Hz rows outside the H x layer,
    // Dy rows outside the E x layer
    const bool lean = C.wr == WROWS && ib >= 1 && last + 1 <= S.nx - 2 && ib >= S.xband[0] &&
                      last < S.xband[1] &&
                      ib >= S.xband[2] && last + 1 < S.xband[3] && S.cond_d1[0] == nullptr &&
                      S.n_poles == 0 && S.n_poles_y == 0 && S.mag_h1[0] == nullptr &&
                      !(EXT && S.cut_y && w.z == 0);
    if (lean) {
        const int jb = w.z + 4 * threadIdx.x;
        const bool yb = jb < S.pitch &&
                        (band4(jb, S.yband[0], S.yband[1]) || band4(jb, S.yband[2], S.yband[3]) ||
                         (threadIdx.x == 31 && in_band(jb + 4, S.yband[2], S.yband[3])));
        if (!__any_sync(0xffffffffu, yb)) {
#pragma unroll 1
            for (int h = 0; h < WROWS; h += 2) te_rows<2, false>(S, ib + h, w.z, C, T.lines, T.nl);
        } else {
#pragma unroll 1
            for (int h = 0; h < WROWS; h += 2) te_rows<2, true>(S, ib + h, w.z, C, T.lines, T.nl);
        }
        return;
    }
#pragma unroll 1
    for (int r = 0; r < C.wr; ++r) {
        if (ib + r >= S.nx) break;
        te_tile<EXT>(S, ib + r, w.z, C, T.lines, T.nl);
    }
}

}  // namespace mtb

#include "yee2d_te3.cuh"

namespace mtb {

}  // namespace mtb

#include "yee2d_tb.cuh"
#include "yee2d_cl.cuh"

using namespace mtb;

struct mtb_yee2d_plan {
    int n_structs = 0;
    DevBuf structs_d, work_d, amp_d, err_d;
    PinnedPair amp_h;
    int n_work = 0;
    int n_work_tm = 0;                 // work items [0, n_work_tm) are TM, the rest TE
    int n_cols = 0;
    int rows = 32;
    int variant = 2;                   // 1 row march, 2 tiles
    bool mpoles = false;               // a structure has magnetic Lorentz poles
    int n_work_te3 = 0;                // the last work items: three-pass TE structures
    bool te_nl = false;                // a three-pass TE structure has chi2 / chi3
    int wr = 1;                        // tiles: rows per warp
    bool ext = false;                  // a structure has conductivity or poles
    bool poles = false;                // a structure has poles (no graph replay)
    int pst = 0;                       // pole buffer holding P(n)
    int graph_mode = 0;                // 0 graphs when eligible, -1 off
    cudaStream_t cap = nullptr;        // private capture stream
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};   // ring flush graph per start parity
    int64_t gkern[2] = {0, 0};         // kernels per graph replay
    DevBuf stage_d;                    // coefficient and phase rows of one flush
    int gend[2] = {0, 1};              // parity after a replay, per start parity
    bool tb = false;                   // temporally blocked kernels after the first step
    bool cl = false;                   // cluster-resident kernel after the first step
    int cl_size = 0, cl_rows = 0;      // CTAs per cluster, rows per CTA
    size_t cl_bytes = 0;               // shared memory per CTA (with the sample staging)
    int cl_nmax = 0, cl_stage = 0;     // steps per launch; line samples staged
    DevBuf tb_work_d, tmaps_d;         // TB tile list (TM first), tensor maps
    DevBuf tb_meta_d, tb_prof_d;       // TB records, padded profiles
    int n_tb_tm = 0, n_tb_te = 0, tb_grid = 148;
    int par = 0;
    int first = 1;
    int64_t last_launches = 0;
    DftState dft;
    LaunchTimer timer;
};

// ---------------------------------------------------------------- TB set-up
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    });
    return fn;
}

// A 2D float32 tensor map over one box array (nx rows x pitch floats), box of
// bc columns x br rows; reads outside the array return zero.
static int tmap_2d(CUtensorMap *m, const float *base, int nx, int pitch, int bc, int br, int s) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
    if (!enc) return fail(MTB_CUDA_ERROR, "cuTensorMapEncodeTiled is not available");
    const cuuint64_t dims[2] = {(cuuint64_t)pitch, (cuuint64_t)nx};
    const cuuint64_t strides[1] = {(cuuint64_t)pitch * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)bc, (cuuint32_t)br};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims,
                           strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(MTB_CUDA_ERROR, "structure %d: tensor map encoding failed (%d)", s, (int)r);
    return MTB_OK;
}

// Structures the TB kernels take: no conductivity, poles, magnetic pairs, PMC
// walls or symmetry cuts (those run on the tile kernels' extended variant).
static bool tb_eligible(const mtb_yee2d_struct &S) {
    return !S.cond_d1[0] && !S.cond_d1[1] && !S.n_poles && !S.n_poles_y && !S.mag_h1[0] &&
           !S.mag_h1[1] && !S.mag_h2[0] && !S.mag_h2[1] && !S.y_pmc && !S.cut_y && !S.cut_x &&
           !S.chi2 && !S.n_mpoles && !S.te3;
}

// Copy n floats of a device array to the host.
static int d2h_floats(std::vector<float> &h, const float *d, int n, int s) {
    h.assign(std::max(n, 0), 0.f);
    if (n <= 0) return MTB_OK;
    const cudaError_t e = cudaMemcpy(h.data(), d, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return fail(MTB_CUDA_ERROR, "structure %d: reading a profile: %s", s,
                    cudaGetErrorString(e));
    return MTB_OK;
}

// Tensor maps, per-structure records (descriptor + line samples), padded
// profiles and the tile list (TM tiles first, then TE) of a TB plan. A
// structure's padded profiles are 4 y rows (hy b, a; ey b, a) of pitch + 128
// floats, column j at index j + 4, then 4 x rows (hx b, a; ex b, a) of
// nx + 32 floats, row i at index i + 4; inert (1, 0) off the arrays.
static int tb_setup_plan(mtb_yee2d_plan *p, const std::vector<mtb_yee2d_struct> &structs) {
    const int n = (int)structs.size();
    std::vector<CUtensorMap> maps((size_t)n * TBM_N);
    std::vector<TbMeta> metas(n);
    std::vector<int64_t> poff(n, 0), xoff(n, 0);
    std::vector<float> prof;
    std::vector<int4> work;
    int rc;
    for (int s = 0; s < n; ++s) {                  // records and padded profiles
        const mtb_yee2d_struct &S = structs[s];
        std::memset(&metas[s], 0, sizeof(TbMeta));
        metas[s].s = S;
        if (S.n_lines > 0) {
            const cudaError_t e = cudaMemcpy(metas[s].lines, S.lines,
                                             sizeof(mtb_line_sample) * S.n_lines,
                                             cudaMemcpyDeviceToHost);
            if (e != cudaSuccess)
                return fail(MTB_CUDA_ERROR, "structure %d: reading line samples: %s", s,
                            cudaGetErrorString(e));
        }
        const int row = S.pitch + 128, xrow = (S.nx + 32 + 3) & ~3;
        poff[s] = (int64_t)prof.size();
        xoff[s] = poff[s] + 4 * (int64_t)row;
        prof.resize(prof.size() + 4 * (size_t)row + 4 * (size_t)xrow);
        float *pp = prof.data() + poff[s], *xp = prof.data() + xoff[s];
        for (int q = 0; q < row; ++q) {
            pp[q] = 1.f; pp[row + q] = 0.f; pp[2 * row + q] = 1.f; pp[3 * row + q] = 0.f;
        }
        for (int q = 0; q < xrow; ++q) {
            xp[q] = 1.f; xp[xrow + q] = 0.f; xp[2 * xrow + q] = 1.f; xp[3 * xrow + q] = 0.f;
        }
        std::vector<float> hb, ha, eb, ea;
        if ((rc = d2h_floats(hb, S.hy_b, S.ny - 1, s)) ||
            (rc = d2h_floats(ha, S.hy_a, S.ny - 1, s)) ||
            (rc = d2h_floats(eb, S.ey_b, S.ny, s)) || (rc = d2h_floats(ea, S.ey_a, S.ny, s)))
            return rc;
        for (int j = 0; j < S.ny - 1; ++j) { pp[j + 4] = hb[j]; pp[row + j + 4] = ha[j]; }
        for (int j = 0; j < S.ny; ++j) { pp[2 * row + j + 4] = eb[j]; pp[3 * row + j + 4] = ea[j]; }
        if ((rc = d2h_floats(hb, S.hx_b, S.nx - 1, s)) ||
            (rc = d2h_floats(ha, S.hx_a, S.nx - 1, s)) ||
            (rc = d2h_floats(eb, S.ex_b, S.nx, s)) || (rc = d2h_floats(ea, S.ex_a, S.nx, s)))
            return rc;
        for (int i = 0; i < S.nx - 1; ++i) { xp[i + 4] = hb[i]; xp[xrow + i + 4] = ha[i]; }
        for (int i = 0; i < S.nx; ++i) { xp[2 * xrow + i + 4] = eb[i]; xp[3 * xrow + i + 4] = ea[i]; }
    }
    for (int pol = 0; pol < 2; ++pol) {
        for (int s = 0; s < n; ++s) {
            const mtb_yee2d_struct &S = structs[s];
            if (S.pol != (pol == 0 ? MTB_TM : MTB_TE)) continue;
            const int nx = S.nx, P = S.pitch;
            CUtensorMap *m = maps.data() + (size_t)s * TBM_N;
            for (int b = 0; b < 2; ++b) {
                if ((rc = tmap_2d(m + TBM_MAIN + b, S.f_main[b], nx, P, TB_C, TB_R, s)) ||
                    (rc = tmap_2d(m + TBM_X + b, S.f_x[b], nx, P, TB_C, TB_R, s)) ||
                    (rc = tmap_2d(m + TBM_Y + b, S.f_y[b], nx, P, TB_C, TB_R, s)) ||
                    (rc = tmap_2d(m + TBM_P1 + b, S.psi[1][b], nx, P, TB_C, TB_R, s)) ||
                    (rc = tmap_2d(m + TBM_P2 + b, S.psi[2][b], nx, P, TB_C, TB_R, s)) ||
                    (rc = tmap_2d(m + TBM_P0W + b, S.psi[0][b], nx, P, TB_C, TB_R, s)) ||
                    (rc = tmap_2d(m + TBM_P3W + b, S.psi[3][b], nx, P, TB_C, TB_R, s)) ||
                    (rc = tmap_2d(m + TBM_P0N + b, S.psi[0][b], nx, P, TB_NARROW, TB_R, s)) ||
                    (rc = tmap_2d(m + TBM_P3N + b, S.psi[3][b], nx, P, TB_NARROW, TB_R, s)))
                    return rc;
            }
            if ((rc = tmap_2d(m + TBM_IEA, S.inv_eps_a, nx, P, TB_C, TB_R, s))) return rc;
            if ((rc = tmap_2d(m + TBM_IEB, S.pol == MTB_TE ? S.inv_eps_b : S.inv_eps_a, nx, P,
                              TB_C, TB_R, s)))
                return rc;
            // layer extents: rows [0, XL) and [XH, nx), columns [0, YL) and [YH, ny)
            const int XL = std::max(S.xband[0], S.xband[2]), XH = std::min(S.xband[1], S.xband[3]);
            const int YL = std::max(S.yband[0], S.yband[2]), YH = std::min(S.yband[1], S.yband[3]);
            const mtb_line_sample *ls = metas[s].lines;
            for (int r0 = 0; r0 < nx; r0 += TB_OUTR) {
                const int wr0 = r0 - TB_T, wr1 = r0 - TB_T + TB_R;
                const bool xl = wr0 < XL || wr1 > XH;
                const int or1 = std::min(r0 + TB_OUTR, nx);
                for (int c0 = 0; c0 < P; c0 += TB_OUTC) {
                    const int wc0 = c0 - 4, wc1 = c0 - 4 + TB_C, oc1 = c0 + TB_OUTC;
                    const int la = std::max(wc0, 0), lb = std::min(wc1, YL);
                    const int ha = std::max(wc0, YH), hb = std::min(wc1, S.ny);
                    const bool lo = lb > la, hi = hb > ha;
                    int flags = xl ? TBF_XPSI : 0;
                    if (lo || hi) {
                        const int a = lo ? la : ha, b = lo ? lb : hb;
                        const int xs = a & ~3;
                        if (lo && hi) {
                            flags |= TBF_YWIDE << TBF_YSHIFT;
                        } else if (b <= xs + TB_NARROW) {
                            flags |= (TBF_YNARROW << TBF_YSHIFT) | ((xs - wc0) << TBF_XS_SHIFT);
                        } else {
                            flags |= TBF_YWIDE << TBF_YSHIFT;
                        }
                    }
                    unsigned lmask = 0;
                    for (int l = 0; l < S.n_lines; ++l) {
                        const mtb_line_sample &q = ls[l];
                        const bool t = q.kind == 0
                                           ? (q.index >= r0 && q.index < or1 && q.lo < oc1 &&
                                              q.hi > c0)
                                           : (q.index >= c0 && q.index < oc1 && q.lo < or1 &&
                                              q.hi > r0);
                        if (t) lmask |= 1u << l;
                    }
                    flags |= (int)(lmask << TBF_LINE_SHIFT);
                    if (!xl && !(lo || hi) && wr0 >= 1 && wr1 <= nx - 1 && wc0 >= 1 &&
                        wc1 <= S.ny - 1)
                        flags |= TBF_LEAN;
                    const int64_t yo = poff[s] + c0, xo = xoff[s] + r0;
                    const int meta_bytes = (int)(sizeof(mtb_yee2d_struct) +
                                                 S.n_lines * sizeof(mtb_line_sample));
                    work.push_back(make_int4(s, r0, c0, flags));
                    work.push_back(make_int4(meta_bytes, S.pitch + 128, (int)(uint32_t)yo,
                                             (int)(yo >> 32)));
                    work.push_back(make_int4((int)(uint32_t)xo, (int)(xo >> 32),
                                             (S.nx + 32 + 3) & ~3, 0));
                }
            }
        }
        if (pol == 0) p->n_tb_tm = (int)(work.size() / TB_WORK);
    }
    p->n_tb_te = (int)(work.size() / TB_WORK) - p->n_tb_tm;
    if ((rc = p->tmaps_d.ensure(sizeof(CUtensorMap) * maps.size())) ||
        (rc = p->tb_work_d.ensure(sizeof(int4) * std::max<size_t>(work.size(), 1))) ||
        (rc = p->tb_meta_d.ensure(sizeof(TbMeta) * metas.size())) ||
        (rc = p->tb_prof_d.ensure(sizeof(float) * prof.size())))
        return rc;
    cudaError_t e = cudaMemcpy(p->tmaps_d.p, maps.data(), sizeof(CUtensorMap) * maps.size(),
                               cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !work.empty())
        e = cudaMemcpy(p->tb_work_d.p, work.data(), sizeof(int4) * work.size(),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(p->tb_meta_d.p, metas.data(), sizeof(TbMeta) * metas.size(),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(p->tb_prof_d.p, prof.data(), sizeof(float) * prof.size(),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_tb_tm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tb_smem<false>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_tb_te, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tb_smem<true>());
    int dev = 0, sms = 0;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail(MTB_CUDA_ERROR, "TB set-up: %s", cudaGetErrorString(e));
    p->tb_grid = std::max(sms, 1);
    p->tb = true;
    return MTB_OK;
}


static int check_ptr(const void *p, const char *what, int s) {
    if (!p) return fail(MTB_INVALID_ARG, "structure %d: %s is null", s, what);
    if (reinterpret_cast<uintptr_t>(p) & 15)
        return fail(MTB_INVALID_ARG, "structure %d: %s is not 16-byte aligned", s, what);
    return MTB_OK;
}

// Fill row_lo / row_hi of a cell list from its row pointer (device -> host).
static int cell_rows(mtb_cells &cl, int rows, int s) {
    cl.row_lo = 1;
    cl.row_hi = 0;
    if (cl.n <= 0) return MTB_OK;
    std::vector<int32_t> rp(rows + 1);
    cudaError_t e = cudaMemcpy(rp.data(), cl.row_ptr, sizeof(int32_t) * (rows + 1),
                               cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return fail(MTB_CUDA_ERROR, "structure %d: reading source rows: %s", s,
                    cudaGetErrorString(e));
    if (rp[0] != 0 || rp[rows] != cl.n)
        return fail(MTB_INVALID_ARG, "structure %d: source row_ptr does not cover %d cells", s,
                    cl.n);
    for (int r = 0; r < rows; ++r) {
        if (rp[r + 1] < rp[r]) return fail(MTB_INVALID_ARG, "structure %d: row_ptr decreasing", s);
        if (rp[r + 1] > rp[r]) {
            if (cl.row_lo > cl.row_hi) cl.row_lo = r;
            cl.row_hi = r;
        }
    }
    // the kernels binary-search a row's columns: they must ascend within each row
    std::vector<int32_t> cv(cl.n);
    e = cudaMemcpy(cv.data(), cl.col, sizeof(int32_t) * cl.n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return fail(MTB_CUDA_ERROR, "structure %d: reading source columns: %s", s,
                    cudaGetErrorString(e));
    for (int r = 0; r < rows; ++r)
        for (int q = rp[r] + 1; q < rp[r + 1]; ++q)
            if (cv[q] < cv[q - 1])
                return fail(MTB_INVALID_ARG, "structure %d: source columns of row %d are not in "
                            "ascending order", s, r);
    return MTB_OK;
}

// Rows where an x profile may be active, conservatively: [0, lo_end) holds
// every active node (a != 0 or b != 1) of the low half, [hi_begin, n) every
// active node of the high half. Inert nodes inside a band are harmless (their
// CPML memory stays zero and the effective derivative is the plain one).
static int profile_band(const float *b_d, const float *a_d, int n, int32_t &lo_end,
                        int32_t &hi_begin, int s) {
    std::vector<float> b(n), a(n);
    cudaError_t e = cudaMemcpy(b.data(), b_d, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(a.data(), a_d, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return fail(MTB_CUDA_ERROR, "structure %d: reading CPML profile: %s", s,
                    cudaGetErrorString(e));
    const int half = n / 2;
    lo_end = 0;
    for (int i = 0; i < half; ++i)
        if (a[i] != 0.f || b[i] != 1.f) lo_end = i + 1;
    hi_begin = n;
    for (int i = n - 1; i >= half; --i)
        if (a[i] != 0.f || b[i] != 1.f) hi_begin = i;
    return MTB_OK;
}

static size_t smem_tm() { return sizeof(WarpSmem<4>) * WARPS2D; }
static size_t smem_te() { return sizeof(WarpSmem<5>) * WARPS2D; }

extern "C" {

static int cl_setup_plan(mtb_yee2d_plan *p, const std::vector<mtb_yee2d_struct> &structs,
                         bool must);


int mtb_yee2d_plan_create(const mtb_yee2d_struct *structs_in, int32_t n,
                          const mtb_dft_region *regions, int32_t n_regions,
                          const mtb_phase_group *groups, int32_t n_groups,
                          int64_t ring_slot_elems, int32_t n_amp_cols, const mtb_tuning *tuning,
                          mtb_yee2d_plan **out) {
    if (!out) return fail(MTB_INVALID_ARG, "out is null");
    *out = nullptr;
    if (n < 1 || !structs_in) return fail(MTB_INVALID_ARG, "need at least one structure");
    if (n_amp_cols < 0) return fail(MTB_INVALID_ARG, "n_amp_cols < 0");
    // default (0) and variant 3: the temporally blocked kernels after the first
    // step when every structure is eligible, else tiles; 2: tiles only
    const int tv = tuning ? tuning->variant : 0;
    if (tv < 0 || tv > 4) return fail(MTB_INVALID_ARG, "2D variant %d not in 0..4", tv);
    const int variant = tv == 1 ? 1 : 2;
    bool want_tb = tv == 3 || tv == 0;
    bool want_cl = tv == 4 || tv == 0;
    int rows = (tuning && tuning->rows_per_warp > 0) ? tuning->rows_per_warp : 32;
    int wr = 1;
    if (variant == 2) {
        // rows per warp: WROWS (register-blocked lean rows) when the batch still
        // fills the GPU with 2 blocks per SM, else one (small, L2-resident
        // batches need the parallelism more than the amortisation)
        int64_t blocks = 0;
        for (int s = 0; s < n; ++s)
            blocks += (int64_t)((structs_in[s].nx + TILE_ROWS - 1) / TILE_ROWS) *
                      ((structs_in[s].pitch + 127) / 128);
        wr = (tuning && tuning->rows_per_warp > 0)
                 ? (tuning->rows_per_warp >= WROWS ? WROWS : 1)
                 : (blocks >= TILE_MIN_BLOCKS ? WROWS : 1);
        rows = TROWS * wr;
    }
    int slots = (tuning && tuning->ring_slots > 0) ? tuning->ring_slots : 32;
    if (ring_slot_elems < 0 || (ring_slot_elems & 3))
        return fail(MTB_INVALID_ARG, "ring_slot_elems must be a non-negative multiple of 4");
    std::vector<mtb_yee2d_struct> structs(structs_in, structs_in + n);
    int64_t n_work = 0;
    for (int s = 0; s < n; ++s) {
        mtb_yee2d_struct &S = structs[s];
        if (S.pol != MTB_TM && S.pol != MTB_TE)
            return fail(MTB_INVALID_ARG, "structure %d: pol must be MTB_TM or MTB_TE", s);
        if (S.nx < 3 || S.ny < 3)
            return fail(MTB_INVALID_ARG, "structure %d: nx, ny must be >= 3 (got %d, %d)", s, S.nx,
                        S.ny);
        if (S.pitch < S.ny || (S.pitch & 3))
            return fail(MTB_INVALID_ARG, "structure %d: pitch %d must be >= ny and a multiple of 4",
                        s, S.pitch);
        if ((int64_t)S.nx * S.pitch >= (1LL << 31))
            return fail(MTB_UNSUPPORTED, "structure %d: grid too large", s);
        if (!(S.dt > 0.f) || !(S.dx > 0.f))
            return fail(MTB_INVALID_ARG, "structure %d: dt, dx must be > 0", s);
        if (S.pol == MTB_TE && S.y_pmc)
            return fail(MTB_UNSUPPORTED, "structure %d: y_pmc is a TM option", s);
        int rc;
        if (S.te3) {
            if (S.pol != MTB_TE || S.te3 != 1)
                return fail(MTB_INVALID_ARG, "structure %d: te3 is a TE flag (0 or 1)", s);
            if (variant != 2)
                return fail(MTB_UNSUPPORTED, "structure %d: tensor eps / oriented poles need "
                            "the tile kernels (variant 2)", s);
            if (S.cut_y || S.cut_x)
                return fail(MTB_UNSUPPORTED, "structure %d: tensor eps / oriented poles with "
                            "symmetry cuts", s);
            if ((rc = check_ptr(S.e_x, "e_x", s)) || (rc = check_ptr(S.e_y, "e_y", s)))
                return rc;
            const bool t = S.tinv[0] || S.tinv[1] || S.tinv[2] || S.tinv[3];
            for (int k = 0; t && k < 4; ++k)
                if ((rc = check_ptr(S.tinv[k], "tinv", s))) return rc;
            const bool nlt = S.nlx[0] || S.nlx[1] || S.nlx[2] || S.nly[0] || S.nly[1] ||
                             S.nly[2];
            if (nlt && t)
                return fail(MTB_UNSUPPORTED, "structure %d: TE chi2 / chi3 with the tensor eps",
                            s);
            for (int k = 0; nlt && k < 3; ++k)
                if ((rc = check_ptr(S.nlx[k], "nlx", s)) || (rc = check_ptr(S.nly[k], "nly", s)))
                    return rc;
            for (int k = 0; nlt && k < 2; ++k)
                if ((rc = check_ptr(S.e_t[k], "e_t", s))) return rc;
            if ((S.c3xy && (!S.n_poles || (rc = check_ptr(S.c3xy, "c3xy", s)))) ||
                (S.c3yx && (!S.n_poles_y || (rc = check_ptr(S.c3yx, "c3yx", s)))))
                return rc ? rc : fail(MTB_INVALID_ARG, "structure %d: cross drives without "
                                      "poles", s);
        } else if (S.tinv[0] || S.c3xy || S.c3yx || S.nlx[0] || S.nly[0]) {
            return fail(MTB_INVALID_ARG, "structure %d: tensor arrays need te3 = 1", s);
        }
        if (S.n_mpoles) {
            if (S.n_mpoles < 0 || S.n_mpoles > MTB_MAX_POLES)
                return fail(MTB_INVALID_ARG, "structure %d: %d magnetic poles outside [0, %d]",
                            s, S.n_mpoles, MTB_MAX_POLES);
            if (S.pol != MTB_TM)
                return fail(MTB_INVALID_ARG, "structure %d: magnetic poles are a TM option", s);
            if (variant != 2)
                return fail(MTB_UNSUPPORTED, "structure %d: magnetic poles need the tile "
                            "kernels (variant 2)", s);
            if (S.mag_h1[0] || S.mag_h1[1] || S.mag_h2[0] || S.mag_h2[1] || S.cut_y == 2 ||
                S.cut_x == 2)
                return fail(MTB_UNSUPPORTED, "structure %d: magnetic poles with magnetic "
                            "conductivity or a live symmetry-cut line", s);
            for (int c = 0; c < 2; ++c) {
                for (int b = 0; b < 2; ++b)
                    if ((rc = check_ptr(S.f_b[c][b], "f_b", s))) return rc;
                for (int b = 0; b < 3; ++b)
                    if ((rc = check_ptr(S.mpol[c][b], "mpol", s)) ||
                        (rc = check_ptr(S.mpc[c][b], "mpc", s)))
                        return rc;
            }
            if ((int64_t)S.n_mpoles * S.nx * S.pitch >= (1LL << 31))
                return fail(MTB_UNSUPPORTED, "structure %d: magnetic pole planes too large", s);
        }
        if (S.chi2 || S.chi3 || S.eps_nl) {
            if (S.pol != MTB_TM)
                return fail(MTB_UNSUPPORTED, "structure %d: chi2 / chi3 on the kernels are TM "
                            "only", s);
            if (variant != 2)
                return fail(MTB_UNSUPPORTED, "structure %d: chi2 / chi3 need the tile kernels "
                            "(variant 2)", s);
            if ((rc = check_ptr(S.chi2, "chi2", s)) || (rc = check_ptr(S.chi3, "chi3", s)) ||
                (rc = check_ptr(S.eps_nl, "eps_nl", s)))
                return rc;
        }
        if (S.cut_y || S.cut_x) {
            if (S.cut_y < 0 || S.cut_y > 2 || S.cut_x < 0 || S.cut_x > 2)
                return fail(MTB_INVALID_ARG, "structure %d: cut_y / cut_x must be 0, 1 or 2", s);
            if (variant != 2)
                return fail(MTB_UNSUPPORTED, "structure %d: symmetry cuts need the tile kernels "
                            "(variant 2)", s);
            if (S.y_pmc)
                return fail(MTB_INVALID_ARG, "structure %d: symmetry cuts and y_pmc exclude "
                            "each other", s);
            if (S.pol == MTB_TE && (S.cut_y == 2 || S.cut_x == 2))
                return fail(MTB_INVALID_ARG, "structure %d: TE cuts are 0 or 1", s);
            for (int a = 0; a < 2; ++a) {
                const int cut = a ? S.cut_x : S.cut_y, map = a ? S.cut_map_x : S.cut_map_y;
                const float ph = a ? S.cut_ph_x : S.cut_ph_y;
                if (cut != 2) continue;
                if (map < 0 || map > 2 || (a == 1 && map == 1) || (ph != 1.f && ph != -1.f))
                    return fail(MTB_INVALID_ARG, "structure %d: cut map %d / phase %g", s, map,
                                (double)ph);
                if (map == 2 && S.nx != S.ny)
                    return fail(MTB_INVALID_ARG, "structure %d: Rotate4 needs a square grid", s);
                for (int b = 0; b < 2; ++b)
                    if ((rc = check_ptr(a ? S.f_y0[b] : S.f_x0[b], "f_x0 / f_y0", s))) return rc;
                // the on-plane H line carries no magnetic pair (core/coeffs.py:240-244)
                if (S.mag_h1[a ? 1 : 0] || S.mag_h2[a ? 1 : 0])
                    return fail(MTB_UNSUPPORTED, "structure %d: a live on-plane H line with "
                                "magnetic conductivity / permeability", s);
            }
        }
        for (int b = 0; b < 2; ++b) {
            if ((rc = check_ptr(S.f_main[b], "f_main", s))) return rc;
            if ((rc = check_ptr(S.f_x[b], "f_x", s))) return rc;
            if ((rc = check_ptr(S.f_y[b], "f_y", s))) return rc;
            for (int k = 0; k < 4; ++k)
                if ((rc = check_ptr(S.psi[k][b], "psi", s))) return rc;
        }
        if ((rc = check_ptr(S.inv_eps_a, "inv_eps_a", s))) return rc;
        const int n_cond = S.pol == MTB_TE ? 2 : 1;
        if (S.cond_d1[0] || S.cond_d1[1]) {
            if (variant != 2)
                return fail(MTB_UNSUPPORTED, "structure %d: conductivity needs the tile "
                            "kernels (variant 2)", s);
            for (int k = 0; k < n_cond; ++k) {
                if ((rc = check_ptr(S.cond_d1[k], "cond_d1", s))) return rc;
                if ((rc = check_ptr(S.cond_d2[k], "cond_d2", s))) return rc;
            }
            if (S.pol == MTB_TM && (S.cond_d1[1] || S.cond_d2[1]))
                return fail(MTB_INVALID_ARG, "structure %d: TM conductivity uses slot 0 only", s);
        } else if (S.cond_d2[0] || S.cond_d2[1]) {
            return fail(MTB_INVALID_ARG, "structure %d: cond_d2 without cond_d1", s);
        }
        for (int k = 0; k < 2; ++k) {
            if (!S.mag_h1[k] && !S.mag_h2[k]) continue;
            if (k == 1 && S.pol == MTB_TE)
                return fail(MTB_INVALID_ARG, "structure %d: TE magnetic pairs use slot 0 only",
                            s);
            if (variant != 2)
                return fail(MTB_UNSUPPORTED, "structure %d: magnetic conductivity needs the "
                            "tile kernels (variant 2)", s);
            if ((rc = check_ptr(S.mag_h1[k], "mag_h1", s))) return rc;
            if ((rc = check_ptr(S.mag_h2[k], "mag_h2", s))) return rc;
        }
        for (int a = 0; a < 2; ++a) {
            const int np = a ? S.n_poles_y : S.n_poles;
            if (np < 0 || np > MTB_MAX_POLES)
                return fail(MTB_INVALID_ARG, "structure %d: %d poles outside [0, %d]", s, np,
                            MTB_MAX_POLES);
            if (np == 0) continue;
            if (a == 1 && S.pol != MTB_TE)
                return fail(MTB_INVALID_ARG, "structure %d: n_poles_y is a TE field", s);
            if (variant != 2)
                return fail(MTB_UNSUPPORTED, "structure %d: poles need the tile kernels "
                            "(variant 2)", s);
            float *const *pp = a ? S.pol_py : S.pol_p;
            const float *const *pc = a ? S.pol_cy : S.pol_c;
            for (int b = 0; b < 3; ++b)
                if ((rc = check_ptr(pp[b], "pole planes", s))) return rc;
            for (int k = 0; k < 3; ++k)
                if ((rc = check_ptr(pc[k], "pole coefficients", s))) return rc;
            if ((int64_t)np * S.nx * S.pitch >= (1LL << 31))
                return fail(MTB_UNSUPPORTED, "structure %d: pole planes too large", s);
        }
        if (S.pol == MTB_TE && (rc = check_ptr(S.inv_eps_b, "inv_eps_b", s))) return rc;
        if (S.pol == MTB_TM && S.explicit_e && (rc = check_ptr(S.e_explicit, "e_explicit", s)))
            return rc;
        if (!S.hx_b || !S.hx_a || !S.hy_b || !S.hy_a || !S.ex_b || !S.ex_a || !S.ey_b || !S.ey_a)
            return fail(MTB_INVALID_ARG, "structure %d: null CPML profile", s);
        mtb_cells *cl[3] = {&S.src_e, &S.src_h1, &S.src_h2};
        for (int c = 0; c < 3; ++c) {
            if (cl[c]->n < 0) return fail(MTB_INVALID_ARG, "structure %d: negative cell count", s);
            if (cl[c]->n > 0 && (!cl[c]->row_ptr || !cl[c]->col || !cl[c]->w ||
                                 cl[c]->amp_col < 0 || cl[c]->amp_col >= n_amp_cols))
                return fail(MTB_INVALID_ARG, "structure %d: source list %d has null arrays or "
                            "amp_col out of [0, %d)", s, c, n_amp_cols);
            if ((rc = cell_rows(*cl[c], S.nx, s))) return rc;
        }
        if (S.pol == MTB_TE && S.src_h2.n > 0)
            return fail(MTB_INVALID_ARG, "structure %d: TE has no second magnetic source", s);
        if (S.n_lines < 0 || S.n_lines > MAXL)
            return fail(MTB_UNSUPPORTED, "structure %d: %d line samples (max %d)", s, S.n_lines,
                        MAXL);
        if (S.n_lines > 0 && !S.lines)
            return fail(MTB_INVALID_ARG, "structure %d: null line sample array", s);
        if (S.n_lines > 0) {
            mtb_line_sample ls[MAXL];
            cudaError_t e = cudaMemcpy(ls, S.lines, sizeof(mtb_line_sample) * S.n_lines,
                                       cudaMemcpyDeviceToHost);
            if (e != cudaSuccess)
                return fail(MTB_CUDA_ERROR, "structure %d: reading line samples: %s", s,
                            cudaGetErrorString(e));
            for (int l = 0; l < S.n_lines; ++l) {
                const mtb_line_sample &q = ls[l];
                const int along = q.kind == 0 ? S.ny : S.nx, across = q.kind == 0 ? S.nx : S.ny;
                if (q.comp < 0 || q.comp > 2 || (q.kind != 0 && q.kind != 1) || q.index < 0 ||
                    q.index >= across || q.lo < 0 || q.hi > along || q.lo >= q.hi ||
                    q.ring_off < 0 || q.ring_off + (q.hi - q.lo) > ring_slot_elems)
                    return fail(MTB_INVALID_ARG, "structure %d: line sample %d out of range", s, l);
            }
        }
        for (int c = 0; c < 3; ++c) {
            const int64_t o = S.ring_full[c];
            if (o >= 0 && ((o & 3) || o + (int64_t)S.nx * S.pitch > ring_slot_elems))
                return fail(MTB_INVALID_ARG, "structure %d: full-grid ring offset %lld invalid", s,
                            (long long)o);
        }
        if ((rc = profile_band(S.hx_b, S.hx_a, S.nx - 1, S.xband[0], S.xband[1], s))) return rc;
        if ((rc = profile_band(S.ex_b, S.ex_a, S.nx, S.xband[2], S.xband[3], s))) return rc;
        if ((rc = profile_band(S.hy_b, S.hy_a, S.ny - 1, S.yband[0], S.yband[1], s))) return rc;
        if ((rc = profile_band(S.ey_b, S.ey_a, S.ny, S.yband[2], S.yband[3], s))) return rc;
        n_work += (int64_t)((S.nx + rows - 1) / rows) * ((S.pitch + 127) / 128);
    }
    if (n_work > (1LL << 30)) return fail(MTB_INVALID_ARG, "batch too large");
    mtb_yee2d_plan *p = new mtb_yee2d_plan();
    p->n_structs = n;
    p->rows = rows;
    p->variant = variant;
    p->wr = wr;
    p->graph_mode = (tuning && tuning->graph < 0) ? -1 : 0;
    p->n_cols = n_amp_cols;
    p->n_work = (int)n_work;
    for (int s = 0; s < n; ++s)
    {
        if (structs[s].cond_d1[0] || structs[s].n_poles > 0 || structs[s].n_poles_y > 0 ||
            structs[s].mag_h1[0] || structs[s].mag_h1[1] || structs[s].cut_y || structs[s].cut_x ||
            structs[s].chi2 || structs[s].n_mpoles || structs[s].te3)
            p->ext = true;
        if (structs[s].n_poles > 0 || structs[s].n_poles_y > 0 || structs[s].n_mpoles > 0)
            p->poles = true;
        if (structs[s].n_mpoles > 0) p->mpoles = true;
        if (structs[s].te3 && structs[s].nlx[0]) p->te_nl = true;
    }
    for (int s = 0; s < n; ++s) want_tb = want_tb && tb_eligible(structs[s]);
    for (int s = 0; s < n; ++s)
        want_cl = want_cl && structs[s].pol == MTB_TM && tb_eligible(structs[s]);
    int rc = p->dft.init(regions, n_regions, groups, n_groups, ring_slot_elems, slots);
    if (!rc) rc = p->structs_d.ensure(sizeof(mtb_yee2d_struct) * n);
    if (!rc) rc = p->work_d.ensure(sizeof(int4) * n_work);
    if (!rc) rc = p->err_d.ensure(sizeof(int));
    if (!rc) {
        cudaError_t e = cudaFuncSetAttribute(k_yee2d_tm<false>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem_tm());
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_yee2d_tm<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem_tm());
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_yee2d_te, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem_te());
        if (e != cudaSuccess)
            rc = fail(MTB_CUDA_ERROR, "shared memory attribute: %s", cudaGetErrorString(e));
    }
    if (rc) { p->dft.release(); delete p; return rc; }
    std::vector<int4> work;
    work.reserve(n_work);
    size_t te3_start = 0;
    for (int pol = 0; pol < 3; ++pol) {
        if (pol == 1) p->n_work_tm = (int)work.size();
        if (pol == 2) te3_start = work.size();
        for (int s = 0; s < n; ++s) {
            if (structs[s].pol != (pol == 0 ? MTB_TM : MTB_TE)) continue;
            if (pol > 0 && (structs[s].te3 != 0) != (pol == 2)) continue;
            for (int i0 = 0; i0 < structs[s].nx; i0 += rows)
                for (int c0 = 0; c0 < structs[s].pitch; c0 += 128)
                    work.push_back(variant == 1
                                       ? make_int4(s, i0, std::min(i0 + rows, structs[s].nx), c0)
                                       : make_int4(s, i0, c0, 0));
        }
    }
    p->n_work_te3 = (int)(work.size() - te3_start);
    cudaError_t e = cudaMemcpy(p->structs_d.p, structs.data(), sizeof(mtb_yee2d_struct) * n,
                               cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(p->work_d.p, work.data(), sizeof(int4) * n_work, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(p->err_d.p, 0, sizeof(int));
    if (e != cudaSuccess) {
        p->dft.release();
        delete p;
        return fail(MTB_CUDA_ERROR, "plan upload failed: %s", cudaGetErrorString(e));
    }
    if (want_cl && (rc = cl_setup_plan(p, structs, tv == 4))) {
        mtb_yee2d_plan_destroy(p);
        return rc;
    }
    if (want_tb && !p->cl && (rc = tb_setup_plan(p, structs))) {
        mtb_yee2d_plan_destroy(p);
        return rc;
    }
    *out = p;
    return MTB_OK;
}

int mtb_yee2d_check(mtb_yee2d_plan *p, void *stream) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    int flag = 0;
    MTB_CUDA_TRY(cudaMemcpyAsync(&flag, p->err_d.p, sizeof(int), cudaMemcpyDeviceToHost,
                                 (cudaStream_t)stream));
    MTB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    if (flag)
        return fail(MTB_DEVICE_TIMEOUT, "a bounded wait for a staged row copy expired on the "
                    "device; the affected steps are incomplete");
    return MTB_OK;
}

// One step's kernels on `st`.
static int launch_step(mtb_yee2d_plan *p, const Ctx2D &C, cudaStream_t st) {
    const int n_tm = p->n_work_tm, n_te = p->n_work - p->n_work_tm;
    const mtb_yee2d_struct *SS = p->structs_d.as<mtb_yee2d_struct>();
    const int4 *W = p->work_d.as<int4>();
    if (p->variant == 2) {
        const dim3 blk(32, TROWS);
        if (n_tm > 0) {
            if (p->mpoles) {
                // magnetic Lorentz poles: their own instantiation (more live registers)
                if (C.first)
                    k_tile_tm<true, true, true><<<n_tm, blk, 0, st>>>(SS, W, n_tm, C);
                else
                    k_tile_tm<false, true, true><<<n_tm, blk, 0, st>>>(SS, W, n_tm, C);
            } else if (C.first && p->ext)
                k_tile_tm<true, true><<<n_tm, blk, 0, st>>>(SS, W, n_tm, C);
            else if (C.first)
                k_tile_tm<true, false><<<n_tm, blk, 0, st>>>(SS, W, n_tm, C);
            else if (p->ext)
                k_tile_tm<false, true><<<n_tm, blk, 0, st>>>(SS, W, n_tm, C);
            else
                k_tile_tm<false, false><<<n_tm, blk, 0, st>>>(SS, W, n_tm, C);
            MTB_CHECK_LAUNCH();
            ++p->last_launches;
        }
        const int n_t3 = p->n_work_te3, n_te1 = n_te - n_t3;
        if (n_te1 > 0) {
            if (p->ext)
                k_tile_te<true><<<n_te1, blk, 0, st>>>(SS, W + n_tm, n_te1, C);
            else
                k_tile_te<false><<<n_te1, blk, 0, st>>>(SS, W + n_tm, n_te1, C);
            MTB_CHECK_LAUNCH();
            ++p->last_launches;
        }
        if (n_t3 > 0) {
            // tensor eps / oriented poles: D and poles, E, Hz as three launches
            const int4 *W3 = W + n_tm + n_te1;
            k_te3<0><<<n_t3, blk, 0, st>>>(SS, W3, n_t3, C);
            MTB_CHECK_LAUNCH();
            k_te3<1><<<n_t3, blk, 0, st>>>(SS, W3, n_t3, C);
            MTB_CHECK_LAUNCH();
            if (p->te_nl) {                    // chi2 / chi3: three Jacobi sweeps
                k_te3<3><<<n_t3, blk, 0, st>>>(SS, W3, n_t3, C);
                MTB_CHECK_LAUNCH();
                k_te3<4><<<n_t3, blk, 0, st>>>(SS, W3, n_t3, C);
                MTB_CHECK_LAUNCH();
                k_te3<5><<<n_t3, blk, 0, st>>>(SS, W3, n_t3, C);
                MTB_CHECK_LAUNCH();
                p->last_launches += 3;
            }
            k_te3<2><<<n_t3, blk, 0, st>>>(SS, W3, n_t3, C);
            MTB_CHECK_LAUNCH();
            p->last_launches += 3;
        }
        return MTB_OK;
    }
    const int blocks_tm = (n_tm + WARPS2D - 1) / WARPS2D;
    const int blocks_te = (n_te + WARPS2D - 1) / WARPS2D;
    if (n_tm > 0) {
        if (C.first)
            k_yee2d_tm<true><<<blocks_tm, 32 * WARPS2D, smem_tm(), st>>>(SS, W, n_tm, C);
        else
            k_yee2d_tm<false><<<blocks_tm, 32 * WARPS2D, smem_tm(), st>>>(SS, W, n_tm, C);
        MTB_CHECK_LAUNCH();
        ++p->last_launches;
    }
    if (n_te > 0) {
        k_yee2d_te<<<blocks_te, 32 * WARPS2D, smem_te(), st>>>(SS, W + n_tm, n_te, C);
        MTB_CHECK_LAUNCH();
        ++p->last_launches;
    }
    return MTB_OK;
}

// out[s * n_off + j] = ring slot s at offset off[j]; offsets outside the slot read 0.
__global__ void k_ring_gather(const float *__restrict__ ring, int64_t slot_elems,
                              const int64_t *__restrict__ off, int n_off, int n_slots,
                              float *__restrict__ out) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= (int64_t)n_off * n_slots) return;
    const int s = (int)(e / n_off), j = (int)(e - (int64_t)s * n_off);
    const int64_t o = off[j];
    out[e] = (o >= 0 && o < slot_elems) ? ring[s * slot_elems + o] : 0.f;
}

// One TB launch pair (TM tiles, then TE tiles) advancing C.nsub steps.
static int launch_tb(mtb_yee2d_plan *p, const TbCtx &C, cudaStream_t st) {
    const CUtensorMap *M = p->tmaps_d.as<CUtensorMap>();
    const int4 *W = p->tb_work_d.as<int4>();
    if (p->n_tb_tm > 0) {
        k_tb_tm<<<std::min(p->tb_grid, p->n_tb_tm), TB_THREADS, tb_smem<false>(), st>>>(
            M, W, p->n_tb_tm, C);
        MTB_CHECK_LAUNCH();
        ++p->last_launches;
    }
    if (p->n_tb_te > 0) {
        k_tb_te<<<std::min(p->tb_grid, p->n_tb_te), TB_THREADS, tb_smem<true>(), st>>>(
            M, W + (size_t)TB_WORK * p->n_tb_tm, p->n_tb_te, C);
        MTB_CHECK_LAUNCH();
        ++p->last_launches;
    }
    return MTB_OK;
}

// Launch context of n TB sub-steps whose first sample goes to ring slot `slot`.
static TbCtx tb_ctx(const mtb_yee2d_plan *p, const float *amp_e, const float *amp_h, int nc,
                    int n, int slot, int par) {
    TbCtx C;
    C.meta = p->tb_meta_d.as<TbMeta>();
    C.prof = p->tb_prof_d.as<float>();
    C.amp_e = amp_e;
    C.amp_h = amp_h;
    C.ncols = nc;
    C.nsub = n;
    C.ring = p->dft.ring_d.as<float>() + (size_t)slot * p->dft.slot_elems;
    C.slot_elems = p->dft.slot_elems;
    C.err = p->err_d.as<int>();
    C.par = par;
    return C;
}

// Cluster-resident kernel: every structure fits the shared memory of one cluster
// (rows split over its CTAs) and the batch occupies at most one cluster per ~16
// SMs, i.e. a launch-latency-bound plan; asked for explicitly, only the fit counts.
// Not applicable leaves p->cl false (or fails when `must`).
static int cl_setup_plan(mtb_yee2d_plan *p, const std::vector<mtb_yee2d_struct> &structs,
                         bool must) {
    const int n = (int)structs.size();
    int nx = 0, pitch = 0;
    for (const auto &S : structs) {
        nx = std::max(nx, S.nx);
        pitch = std::max(pitch, S.pitch);
    }
    int dev = 0, sms = 0, optin = 0;
    MTB_CUDA_TRY(cudaGetDevice(&dev));
    MTB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MTB_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    // the function attributes once per process (the largest shared memory the device
    // allows), the cluster occupancy once per shared-memory size: plan creation stays cheap
    static std::mutex mu;
    static int size_cached = 0;
    static std::vector<std::pair<size_t, int>> occ_cache;
    std::lock_guard<std::mutex> lock(mu);
    if (!size_cached) {
        size_cached = CL_MAX;
        if (cudaFuncSetAttribute(k_cl_tm, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess) {
            cudaGetLastError();
            size_cached = 8;
        }
        MTB_CUDA_TRY(cudaFuncSetAttribute(k_cl_tm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          optin));
    }
    const int size = size_cached;
    const int rows = (nx + size - 1) / size;
    size_t bytes = cl_smem(rows, pitch);
    const bool fits = bytes <= (size_t)optin && (int64_t)rows * (pitch / 4) <= CL_THREADS;
    // line samples staged in shared memory for a whole launch (written to the ring at its
    // end, so that no global store sits before a cluster barrier): as many steps per
    // launch as the remaining shared memory holds, at most a ring's worth
    int64_t span = 0;
    for (const auto &S : structs) {
        if (S.n_lines <= 0) continue;
        mtb_line_sample ls[MAXL];
        MTB_CUDA_TRY(cudaMemcpy(ls, S.lines, sizeof(mtb_line_sample) * S.n_lines,
                                cudaMemcpyDeviceToHost));
        int64_t lo = 0, hi = 0;
        cl_line_span(ls, S.n_lines, lo, hi);
        span = std::max(span, hi - lo);
    }
    const int G = p->dft.slots;
    int nmax = G, stage = 0;
    if (fits && span > 0) {
        const int64_t room = ((int64_t)optin - (int64_t)bytes) / (int64_t)(sizeof(float) * span);
        if (room >= std::min(G, 8)) {
            nmax = (int)std::min<int64_t>(G, room);
            stage = 1;
            bytes = cl_smem_staged(rows, pitch, span, nmax);
        }
    }
    if (!fits || (!must && (int64_t)n * size > sms)) {
        if (must)
            return fail(MTB_UNSUPPORTED, "cluster kernel: %zu bytes of shared memory per CTA "
                        "(%d rows x pitch %d) exceed %d", bytes, rows, pitch, optin);
        return MTB_OK;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = size;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(size * n);
    cfg.blockDim = dim3(CL_THREADS);
    cfg.dynamicSmemBytes = bytes;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = -1;
    for (const auto &e : occ_cache)
        if (e.first == bytes) clusters = e.second;
    if (clusters < 0) {
        cfg.gridDim = dim3(size);
        if (cudaOccupancyMaxActiveClusters(&clusters, k_cl_tm, &cfg) != cudaSuccess) {
            cudaGetLastError();
            clusters = 0;
        }
        occ_cache.emplace_back(bytes, clusters);
    }
    if (clusters < 1) {
        if (must) return fail(MTB_UNSUPPORTED, "cluster kernel: no cluster of %d CTAs fits", size);
        return MTB_OK;
    }
    p->cl = true;
    p->cl_size = size;
    p->cl_rows = rows;
    p->cl_bytes = bytes;
    p->cl_nmax = nmax;
    p->cl_stage = stage;
    return MTB_OK;
}

// n cluster-resident steps from parity par; samples from ring slot `slot` on.
static int launch_cl(mtb_yee2d_plan *p, const float *amp_e, const float *amp_h, int nc, int n,
                     int slot, int par, cudaStream_t st) {
    ClCtx C;
    C.structs = p->structs_d.as<mtb_yee2d_struct>();
    C.amp_e = amp_e;
    C.amp_h = amp_h;
    C.ncols = nc;
    C.nsub = n;
    C.ring = p->dft.ring_d.as<float>() + (size_t)slot * p->dft.slot_elems;
    C.slot_elems = p->dft.slot_elems;
    C.par = par;
    C.rows = p->cl_rows;
    C.stage = p->cl_stage;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = p->cl_size;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(p->cl_size * p->n_structs);
    cfg.blockDim = dim3(CL_THREADS);
    cfg.dynamicSmemBytes = p->cl_bytes;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    MTB_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_cl_tm, C));
    MTB_CHECK_LAUNCH();
    ++p->last_launches;
    return MTB_OK;
}

// Capture one ring flush (G steps from parity par0, then the contraction)
// reading its coefficient and phase rows from the plan's staging buffer.
static int build_flush_graph(mtb_yee2d_plan *p, int par0, int nc) {
    const int G = p->dft.slots;
    if (!p->cap) MTB_CUDA_TRY(cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking));
    const float *stage = p->stage_d.as<float>();
    const float *phase = stage + 2 * (size_t)G * nc;
    const int64_t l0 = mtb_launch_count(), ll0 = p->last_launches;
    MTB_CUDA_TRY(cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeThreadLocal));
    int rc = MTB_OK;
    int par = par0;
    for (int s = 0; s < G && !rc;) {
        if (p->cl) {                             // cluster launches of up to cl_nmax steps
            const int n = std::min(p->cl_nmax, G - s);
            rc = launch_cl(p, stage + (size_t)s * nc, stage + (size_t)G * nc + (size_t)s * nc, nc,
                           n, s, par, p->cap);
            par ^= n & 1;
            s += n;
            continue;
        }
        if (p->tb) {                             // TB launches of up to TB_T steps
            const int n = std::min(TB_T, G - s);
            const TbCtx C = tb_ctx(p, stage + (size_t)s * nc,
                                   stage + (size_t)G * nc + (size_t)s * nc, nc, n, s, par);
            rc = launch_tb(p, C, p->cap);
            par ^= 1;
            s += n;
            continue;
        }
        Ctx2D C;
        C.amp_e = stage + (size_t)s * nc;
        C.amp_h = stage + (size_t)G * nc + (size_t)s * nc;
        C.ring = p->dft.ring_d.as<float>() + (size_t)s * p->dft.slot_elems;
        C.err = p->err_d.as<int>();
        C.par = par;
        C.first = 0;
        C.wr = p->wr;
        C.pst = 0;                               // no poles in graph-replayed plans
        rc = launch_step(p, C, p->cap);
        par ^= 1;
        ++s;
    }
    p->gend[par0] = par;
    if (!rc && p->dft.n_regions > 0) {
        rc = p->dft.contract(0, G, p->cap, nullptr, phase);
        if (!rc) ++p->last_launches;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(p->cap, &g);
    const int64_t nk = mtb_launch_count() - l0;
    count_launch(-nk);                           // captured, not launched
    p->last_launches = ll0;
    if (!rc && e != cudaSuccess)
        rc = fail(MTB_CUDA_ERROR, "graph capture: %s", cudaGetErrorString(e));
    if (!rc) {
        const cudaError_t ei = cudaGraphInstantiate(&p->gexec[par0], g, 0);
        if (ei != cudaSuccess) {
            p->gexec[par0] = nullptr;
            rc = fail(MTB_CUDA_ERROR, "graph instantiate: %s", cudaGetErrorString(ei));
        }
    }
    if (g) cudaGraphDestroy(g);
    p->gkern[par0] = nk;
    return rc;
}

int mtb_yee2d_run(mtb_yee2d_plan *p, int64_t t0, int32_t k, const double *coef_e,
                  const double *coef_h, void *stream) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    if (k < 0) return fail(MTB_INVALID_ARG, "k < 0");
    p->last_launches = 0;
    if (k == 0) return MTB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    // the row march's bounded waits may have raised the error flag (the TB kernels' flag
    // is read by mtb_yee2d_check, which the engine calls when it exports the state; the
    // one-step tiles and the cluster kernel never wait)
    if (p->variant == 1 && (rc = mtb_yee2d_check(p, stream))) return rc;
    const int nc = std::max(p->n_cols, 1);
    const size_t per = (size_t)k * nc;
    void *hp = nullptr;
    if ((rc = p->amp_h.acquire(2 * per * sizeof(float), &hp))) return rc;
    if ((rc = p->amp_d.ensure(2 * per * sizeof(float)))) return rc;
    if ((rc = p->dft.upload_phases(t0, k, st))) return rc;
    float *ah = static_cast<float *>(hp);
    for (size_t i = 0; i < per; ++i) {
        ah[i] = coef_e ? (float)coef_e[i] : 0.f;
        ah[per + i] = coef_h ? (float)coef_h[i] : 0.f;
    }
    MTB_CUDA_TRY(cudaMemcpyAsync(p->amp_d.p, ah, 2 * per * sizeof(float),
                                 cudaMemcpyHostToDevice, st));
    if ((rc = p->amp_h.queued(st))) return rc;
    const float *ad = p->amp_d.as<float>();
    const int G = p->dft.slots;
    const size_t prow = (size_t)p->dft.total_nf * 4;         // floats per phase row
    // graph replay keys on the start parity; the pole buffers rotate with period 3
    const bool graphs = p->graph_mode >= 0 && !p->timer.on && G >= 2 && k >= G && !p->poles;
    if (graphs && (rc = p->stage_d.ensure(sizeof(float) * (2 * (size_t)G * nc + G * prow))))
        return rc;
    int slot = 0;
    int s = 0;
    while (s < k) {
        if (graphs && slot == 0 && !p->first && k - s >= G) {
            // one ring flush as a graph replay: stage its rows, launch
            float *stage = p->stage_d.as<float>();
            MTB_CUDA_TRY(cudaMemcpyAsync(stage, ad + (size_t)s * nc, sizeof(float) * G * nc,
                                         cudaMemcpyDeviceToDevice, st));
            MTB_CUDA_TRY(cudaMemcpyAsync(stage + (size_t)G * nc, ad + per + (size_t)s * nc,
                                         sizeof(float) * G * nc, cudaMemcpyDeviceToDevice, st));
            if (prow > 0 && p->dft.n_regions > 0)
                MTB_CUDA_TRY(cudaMemcpyAsync(stage + 2 * (size_t)G * nc,
                                             p->dft.phase_d.as<float>() + (size_t)s * prow,
                                             sizeof(float) * G * prow, cudaMemcpyDeviceToDevice,
                                             st));
            if (!p->gexec[p->par] && (rc = build_flush_graph(p, p->par, nc))) return rc;
            MTB_CUDA_TRY(cudaGraphLaunch(p->gexec[p->par], st));
            count_launch(p->gkern[p->par]);
            p->last_launches += p->gkern[p->par];
            p->par = p->gend[p->par];
            s += G;
            continue;
        }
        if (p->cl && !p->first) {
            // cluster-resident: the rest of the ring in one launch
            const int n = std::min(p->cl_nmax, std::min(G - slot, k - s));
            if ((rc = p->timer.begin(st, 0))) return rc;
            if ((rc = launch_cl(p, ad + (size_t)s * nc, ad + per + (size_t)s * nc, nc, n, slot,
                                p->par, st)))
                return rc;
            if ((rc = p->timer.end(st))) return rc;
            p->par ^= n & 1;
            s += n;
            slot += n;
            if (slot == G || s == k) {
                if (p->dft.n_regions > 0) {
                    if ((rc = p->dft.contract(s - slot, slot, st, &p->timer))) return rc;
                    ++p->last_launches;
                }
                slot = 0;
            }
            continue;
        }
        if (p->tb && !p->first) {
            // TB: up to TB_T steps per launch, never past the ring's end
            const int n = std::min(TB_T, std::min(G - slot, k - s));
            const TbCtx C = tb_ctx(p, ad + (size_t)s * nc, ad + per + (size_t)s * nc, nc, n, slot,
                                   p->par);
            if ((rc = p->timer.begin(st, 0))) return rc;
            if ((rc = launch_tb(p, C, st))) return rc;
            if ((rc = p->timer.end(st))) return rc;
            p->par ^= 1;
            s += n;
            slot += n;
            if (slot == G || s == k) {
                if (p->dft.n_regions > 0) {
                    if ((rc = p->dft.contract(s - slot, slot, st, &p->timer))) return rc;
                    ++p->last_launches;
                }
                slot = 0;
            }
            continue;
        }
        Ctx2D C;
        C.amp_e = ad + (size_t)s * nc;
        C.amp_h = ad + per + (size_t)s * nc;
        C.ring = p->dft.ring_d.as<float>() + (size_t)slot * p->dft.slot_elems;
        C.err = p->err_d.as<int>();
        C.par = p->par;
        C.first = p->first;
        C.wr = p->wr;
        C.pst = p->pst;
        if ((rc = p->timer.begin(st, 0))) return rc;
        if ((rc = launch_step(p, C, st))) return rc;
        if ((rc = p->timer.end(st))) return rc;
        p->par ^= 1;
        p->pst = (p->pst + 1) % 3;
        p->first = 0;
        ++slot;
        if (slot == G || s == k - 1) {
            if (p->dft.n_regions > 0) {
                if ((rc = p->dft.contract(s + 1 - slot, slot, st, &p->timer))) return rc;
                ++p->last_launches;
            }
            slot = 0;
        }
        ++s;
    }
    return p->timer.collect();
}

int mtb_yee2d_set_timing(mtb_yee2d_plan *p, int32_t enable) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    p->timer.on = enable != 0;
    p->timer.ms[0] = p->timer.ms[1] = 0;
    p->timer.count[0] = p->timer.count[1] = 0;
    return MTB_OK;
}

int mtb_yee2d_timing(const mtb_yee2d_plan *p, double *step_ms, int64_t *step_launches,
                     double *dft_ms, int64_t *dft_launches) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    if (step_ms) *step_ms = p->timer.ms[0];
    if (step_launches) *step_launches = p->timer.count[0];
    if (dft_ms) *dft_ms = p->timer.ms[1];
    if (dft_launches) *dft_launches = p->timer.count[1];
    return MTB_OK;
}

int32_t mtb_yee2d_pole_slot(const mtb_yee2d_plan *p) { return p ? p->pst : -1; }

int32_t mtb_yee2d_current(const mtb_yee2d_plan *p) { return p ? p->par : -1; }

int64_t mtb_yee2d_last_launches(const mtb_yee2d_plan *p) { return p ? p->last_launches : -1; }

int mtb_yee2d_ring_gather(const mtb_yee2d_plan *p, const int64_t *offsets, int32_t n_off,
                          int32_t n_slots, float *out, void *stream) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    if (n_off < 0 || n_slots < 0 || n_slots > p->dft.slots)
        return fail(MTB_INVALID_ARG, "ring gather: %d offsets x %d slots (ring of %d)", n_off,
                    n_slots, p->dft.slots);
    if ((int64_t)n_off * n_slots == 0) return MTB_OK;
    if (!offsets || !out || !p->dft.ring_d.p)
        return fail(MTB_INVALID_ARG, "ring gather: null offsets, output or ring");
    const int64_t n = (int64_t)n_off * n_slots;
    k_ring_gather<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        p->dft.ring_d.as<float>(), p->dft.slot_elems, offsets, n_off, n_slots, out);
    MTB_CHECK_LAUNCH();
    return MTB_OK;
}

int mtb_yee2d_ring(const mtb_yee2d_plan *p, float **ring, int64_t *slot_elems, int32_t *slots) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    if (ring) *ring = const_cast<float *>(p->dft.ring_d.as<float>());
    if (slot_elems) *slot_elems = p->dft.slot_elems;
    if (slots) *slots = p->dft.slots;
    return MTB_OK;
}

void mtb_yee2d_plan_destroy(mtb_yee2d_plan *p) {
    if (!p) return;
    for (int q = 0; q < 2; ++q)
        if (p->gexec[q]) cudaGraphExecDestroy(p->gexec[q]);
    if (p->cap) cudaStreamDestroy(p->cap);
    p->stage_d.release();
    p->tb_work_d.release();
    p->tmaps_d.release();
    p->tb_meta_d.release();
    p->tb_prof_d.release();
    p->structs_d.release();
    p->work_d.release();
    p->amp_d.release();
    p->err_d.release();
    p->amp_h.release();
    p->dft.release();
    p->timer.release();
    delete p;
}

}  // extern "C"

// ---------------------------------------------------------------- no-allocation run
// mtb_yee2d_run_noalloc: the plan's scratch (descriptor copy, work list, DFT
// tables, sample ring, error flag) is carved out of one file-scope device
// array instead of cudaMalloc'd buffers; the tables a plan builds on the host
// are built here by small set-up kernels. The step and contraction kernels
// are the plan's own.
namespace mtb {

__global__ void k_dft_contract(const mtb_dft_region *__restrict__ regions,
                               const int *__restrict__ blk_region,
                               const int64_t *__restrict__ blk_start,
                               const int *__restrict__ group_nf, const int *__restrict__ group_off,
                               int total_nf, const float *__restrict__ phase, int row0, int n,
                               const float *__restrict__ ring, int64_t slot_elems);

static __device__ __align__(256) unsigned char g_noalloc_scratch[MTB_NOALLOC_SCRATCH_BYTES];
constexpr int NA_MAX_DEV = 64;
constexpr int NA_MAX_REGIONS = 64;
constexpr int NA_MAX_GROUPS = 16;
constexpr int NA_CT = 256;              // contraction block size (common.cu)
constexpr int NA_ERR_COLS = 1 << 30;    // error-flag bit: source columns out of order
constexpr int NA_ERR_ROWS = 1 << 29;    // error-flag bit: a source row_ptr is malformed
constexpr int NA_ERR_LINES = 1 << 28;   // error-flag bit: a line sample is out of range
// device address of the array, per device, filled once under g_noalloc_mu
static unsigned char *g_noalloc_dev[NA_MAX_DEV];
static std::mutex g_noalloc_mu;

// Checks and derived fields of the descriptor copy (what mtb_yee2d_plan_create
// computes on the host): each source list's row pointer (rp[0] == 0,
// rp[nx] == n, non-decreasing) before any of its columns is read, the column
// order within a row, the line samples against the ring slot, the x-layer
// bands and the source row ranges. Failures set bits of *err; the host reads
// them back before any step kernel runs.
__global__ void k_na_struct(mtb_yee2d_struct *S, int *err, int64_t ring_slot_elems) {
    __shared__ int lh, hh, le, he, rlo[3], rhi[3], bad[3];
    const int nx = S->nx;
    const int nh = nx - 1, ne = nx;
    const mtb_cells *cl[3] = {&S->src_e, &S->src_h1, &S->src_h2};
    if (threadIdx.x == 0) {
        lh = 0; hh = nh; le = 0; he = ne;
        for (int c = 0; c < 3; ++c) {
            rlo[c] = 0x7fffffff; rhi[c] = -1;
            const int n = cl[c]->n;
            bad[c] = n > 0 && (cl[c]->row_ptr[0] != 0 || cl[c]->row_ptr[nx] != n);
        }
    }
    __syncthreads();
    for (int c = 0; c < 3; ++c) {
        const int n = cl[c]->n;
        if (n <= 0) continue;
        for (int r = threadIdx.x; r < nx; r += blockDim.x) {
            const int e0 = cl[c]->row_ptr[r], e1 = cl[c]->row_ptr[r + 1];
            if (e0 < 0 || e1 < e0 || e1 > n) atomicOr(&bad[c], 1);
        }
    }
    for (int l = threadIdx.x; l < S->n_lines; l += blockDim.x) {
        const mtb_line_sample q = S->lines[l];
        const int along = q.kind == 0 ? S->ny : S->nx, across = q.kind == 0 ? S->nx : S->ny;
        if (q.comp < 0 || q.comp > 2 || (q.kind != 0 && q.kind != 1) || q.index < 0 ||
            q.index >= across || q.lo < 0 || q.hi > along || q.lo >= q.hi || q.ring_off < 0 ||
            q.ring_off + (q.hi - q.lo) > ring_slot_elems)
            atomicOr(err, NA_ERR_LINES);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ne; i += blockDim.x) {
        if (i < nh && (S->hx_a[i] != 0.f || S->hx_b[i] != 1.f)) {
            if (i < nh / 2) atomicMax(&lh, i + 1); else atomicMin(&hh, i);
        }
        if (S->ex_a[i] != 0.f || S->ex_b[i] != 1.f) {
            if (i < ne / 2) atomicMax(&le, i + 1); else atomicMin(&he, i);
        }
    }
    for (int c = 0; c < 3; ++c) {
        if (cl[c]->n <= 0) continue;
        if (bad[c]) {                      // columns are only read through a valid row_ptr
            if (threadIdx.x == 0) atomicOr(err, NA_ERR_ROWS);
            continue;
        }
        for (int r = threadIdx.x; r < nx; r += blockDim.x) {
            const int e0 = cl[c]->row_ptr[r], e1 = cl[c]->row_ptr[r + 1];
            if (e1 > e0) {
                atomicMin(&rlo[c], r);
                atomicMax(&rhi[c], r);
            }
            // the kernels binary-search a row's columns: flag a descending pair
            for (int q = e0 + 1; q < e1; ++q)
                if (cl[c]->col[q] < cl[c]->col[q - 1]) {
                    atomicOr(err, NA_ERR_COLS);
                    break;
                }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        S->xband[0] = lh; S->xband[1] = hh; S->xband[2] = le; S->xband[3] = he;
        mtb_cells *w[3] = {&S->src_e, &S->src_h1, &S->src_h2};
        for (int c = 0; c < 3; ++c) {
            if (rhi[c] < 0) { w[c]->row_lo = 1; w[c]->row_hi = 0; }
            else { w[c]->row_lo = rlo[c]; w[c]->row_hi = rhi[c]; }
        }
    }
}

__global__ void k_na_work(int4 *work, int nx, int rows, int nch, int n_work) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_work) return;
    const int seg = e / nch, c = e - seg * nch;
    const int i0 = seg * rows;
    work[e] = make_int4(0, i0, min(i0 + rows, nx), c * 128);
}

__global__ void k_na_blk(int *blk_region, const int64_t *blk_start, int n_regions,
                         int64_t n_blocks) {
    const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= n_blocks) return;
    int r = 0;
    while (r + 1 < n_regions && blk_start[r + 1] <= b) ++r;
    blk_region[b] = r;
}

// phase table rows [0, k) for steps t0 .. t0+k-1, same layout and formulas
// as DftState::upload_phases (FP64 mode 0, reference float32 mode 1)
__global__ void k_na_phase(float *phase, const double *freqs, const int *group_nf,
                           const int *group_off, const double *group_dt, const int *group_mode,
                           int n_groups, int total_nf, int64_t t0, int k) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= (int64_t)k * total_nf) return;
    const int s = (int)(e / total_nf), fi = (int)(e - (int64_t)s * total_nf);
    int g = 0;
    while (g + 1 < n_groups && group_off[g + 1] <= fi) ++g;
    const double dt = group_dt[g], fr = freqs[fi];
    const double two_pi = 6.283185307179586;
    float *p = phase + e * 4;
    for (int h = 0; h < 2; ++h) {
        const double tt = ((double)(t0 + s) + 0.5 * (h + 1)) * dt;
        float c, sn;
        if (group_mode[g] == 0) {
            const double arg = two_pi * fr * tt;
            c = (float)(dt * cos(arg));
            sn = (float)(-dt * sin(arg));
        } else {
            const float arg = ((float)two_pi * (float)fr) * (float)tt;
            c = (float)dt * cosf(arg);
            sn = (float)dt * -sinf(arg);
        }
        p[2 * h] = c;
        p[2 * h + 1] = sn;
    }
}

__global__ void k_na_amp(float *amp, const double *coef, int k, int has_e, int has_h) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= k) return;
    amp[s] = has_e ? (float)coef[s] : 0.f;
    amp[k + s] = has_h ? (float)coef[k + s] : 0.f;
}

static size_t na_align(size_t n) { return (n + 255) & ~(size_t)255; }

}  // namespace mtb

extern "C" int mtb_yee2d_run_noalloc(const mtb_yee2d_struct *s, const mtb_dft_region *regions,
                                     int32_t n_regions, const mtb_phase_group *groups,
                                     int32_t n_groups, int64_t ring_slot_elems,
                                     int32_t ring_slots, int32_t parity, int64_t t0, int32_t k,
                                     const double *coef_e, const double *coef_h, void *stream) {
    using namespace mtb;
    cudaStream_t st = (cudaStream_t)stream;
    if (!s) return fail(MTB_INVALID_ARG, "noalloc: structure is null");
    if (k < 0) return fail(MTB_INVALID_ARG, "noalloc: k < 0");
    if (parity != 0 && parity != 1) return fail(MTB_INVALID_ARG, "noalloc: parity must be 0 or 1");
    const mtb_yee2d_struct &S = *s;
    if (S.pol != MTB_TM && S.pol != MTB_TE)
        return fail(MTB_INVALID_ARG, "noalloc: pol must be MTB_TM or MTB_TE");
    if (S.nx < 3 || S.ny < 3 || S.pitch < S.ny || (S.pitch & 3) ||
        (int64_t)S.nx * S.pitch >= (1LL << 31))
        return fail(MTB_INVALID_ARG, "noalloc: bad extents nx=%d ny=%d pitch=%d", S.nx, S.ny,
                    S.pitch);
    if (!(S.dt > 0.f) || !(S.dx > 0.f)) return fail(MTB_INVALID_ARG, "noalloc: dt, dx must be > 0");
    if (S.pol == MTB_TE && (S.y_pmc || S.src_h2.n > 0))
        return fail(MTB_INVALID_ARG, "noalloc: y_pmc / second magnetic source are TM options");
    if (S.cond_d1[0] || S.cond_d1[1] || S.cond_d2[0] || S.cond_d2[1] || S.n_poles ||
        S.n_poles_y || S.mag_h1[0] || S.mag_h1[1] || S.mag_h2[0] || S.mag_h2[1] || S.cut_y ||
        S.cut_x || S.chi2 || S.n_mpoles || S.te3)
        return fail(MTB_UNSUPPORTED, "noalloc: conductivity, poles and symmetry cuts need the "
                    "tile kernels");
    int rc;
    for (int b = 0; b < 2; ++b) {
        if ((rc = check_ptr(S.f_main[b], "f_main", 0)) || (rc = check_ptr(S.f_x[b], "f_x", 0)) ||
            (rc = check_ptr(S.f_y[b], "f_y", 0)))
            return rc;
        for (int q = 0; q < 4; ++q)
            if ((rc = check_ptr(S.psi[q][b], "psi", 0))) return rc;
    }
    if ((rc = check_ptr(S.inv_eps_a, "inv_eps_a", 0))) return rc;
    if (S.pol == MTB_TE && (rc = check_ptr(S.inv_eps_b, "inv_eps_b", 0))) return rc;
    if (S.pol == MTB_TM && S.explicit_e && (rc = check_ptr(S.e_explicit, "e_explicit", 0)))
        return rc;
    if (!S.hx_b || !S.hx_a || !S.hy_b || !S.hy_a || !S.ex_b || !S.ex_a || !S.ey_b || !S.ey_a)
        return fail(MTB_INVALID_ARG, "noalloc: null CPML profile");
    const mtb_cells *cl[3] = {&S.src_e, &S.src_h1, &S.src_h2};
    for (int c = 0; c < 3; ++c)
        if (cl[c]->n < 0 || (cl[c]->n > 0 && (!cl[c]->row_ptr || !cl[c]->col || !cl[c]->w ||
                                              cl[c]->amp_col != 0)))
            return fail(MTB_INVALID_ARG, "noalloc: source list %d: null arrays or amp_col != 0", c);
    if (S.n_lines < 0 || S.n_lines > MAXL || (S.n_lines > 0 && !S.lines))
        return fail(MTB_INVALID_ARG, "noalloc: bad line sample list");
    if (ring_slots < 1 || ring_slots > 64)
        return fail(MTB_INVALID_ARG, "noalloc: ring_slots must be in [1, 64]");
    if (n_regions == 0 && (S.n_lines > 0 || S.ring_full[0] >= 0 || S.ring_full[1] >= 0 ||
                           S.ring_full[2] >= 0))
        return fail(MTB_INVALID_ARG, "noalloc: samples requested but no DFT region reads them");
    if (ring_slot_elems < 0 || (ring_slot_elems & 3))
        return fail(MTB_INVALID_ARG, "noalloc: ring_slot_elems must be a multiple of 4");
    for (int c = 0; c < 3; ++c) {
        const int64_t o = S.ring_full[c];
        if (o >= 0 && ((o & 3) || o + (int64_t)S.nx * S.pitch > ring_slot_elems))
            return fail(MTB_INVALID_ARG, "noalloc: full-grid ring offset invalid");
    }
    if (n_regions < 0 || n_regions > NA_MAX_REGIONS || n_groups < 0 || n_groups > NA_MAX_GROUPS ||
        (n_regions > 0 && (!regions || !groups)))
        return fail(MTB_INVALID_ARG, "noalloc: at most %d regions and %d phase groups",
                    NA_MAX_REGIONS, NA_MAX_GROUPS);
    // phase groups and region block prefix on the stack (host)
    int gnf[NA_MAX_GROUPS + 1], goff[NA_MAX_GROUPS + 1], gmode[NA_MAX_GROUPS + 1];
    double gdt[NA_MAX_GROUPS + 1];
    int total_nf = 0, maxnf = 1;
    for (int g = 0; g < n_groups; ++g) {
        if (groups[g].nf < 1 || groups[g].nf > 256 || !groups[g].freqs ||
            (groups[g].mode != 0 && groups[g].mode != 1))
            return fail(MTB_INVALID_ARG, "noalloc: phase group %d invalid", g);
        gnf[g] = groups[g].nf;
        goff[g] = total_nf;
        gmode[g] = groups[g].mode;
        gdt[g] = groups[g].dt;
        total_nf += groups[g].nf;
        maxnf = std::max(maxnf, groups[g].nf);
    }
    gnf[n_groups] = goff[n_groups] = gmode[n_groups] = 0;
    gdt[n_groups] = 0.0;
    goff[n_groups] = total_nf;
    int64_t bs[NA_MAX_REGIONS + 1];
    int64_t n_blocks = 0;
    for (int r = 0; r < n_regions; ++r) {
        const mtb_dft_region &R = regions[r];
        if (R.group < 0 || R.group >= n_groups || (R.toff != 1 && R.toff != 2) || R.rows < 0 ||
            R.cols < 0 || !R.acc || R.ring_a < 0 ||
            R.ring_a + (int64_t)(R.rows - 1) * R.ring_pitch + R.cols > ring_slot_elems ||
            (R.ring_b >= 0 && R.ring_b + (int64_t)(R.rows - 1) * R.ring_pitch + R.cols >
                                  ring_slot_elems))
            return fail(MTB_INVALID_ARG, "noalloc: region %d invalid", r);
        bs[r] = n_blocks;
        n_blocks += ((int64_t)R.rows * R.cols + NA_CT - 1) / NA_CT;
    }
    bs[n_regions] = n_blocks;
    const int rows = 32;
    const int nch = (S.pitch + 127) / 128;
    const int n_work = ((S.nx + rows - 1) / rows) * nch;
    // scratch layout
    const size_t fixed = na_align(sizeof(mtb_yee2d_struct)) + 256 +
                         na_align(sizeof(mtb_dft_region) * (n_regions + 1)) +
                         na_align(sizeof(int64_t) * (n_regions + 1)) +
                         4 * na_align(sizeof(double) * (NA_MAX_GROUPS + 1)) +
                         na_align(sizeof(double) * (total_nf + 1)) +
                         na_align(sizeof(int) * (n_blocks + 1)) + na_align(sizeof(int4) * n_work) +
                         (n_regions > 0 ? na_align(sizeof(float) * (size_t)ring_slots *
                                                   ring_slot_elems) : 0);
    int CH = 256;
    auto per_chunk = [&](int ch) {
        return na_align(sizeof(double) * 2 * ch) + na_align(sizeof(float) * 2 * ch) +
               na_align(sizeof(float) * 4 * (size_t)ch * std::max(total_nf, 1));
    };
    while (CH > 1 && fixed + per_chunk(CH) > MTB_NOALLOC_SCRATCH_BYTES) CH /= 2;
    if (fixed + per_chunk(CH) > MTB_NOALLOC_SCRATCH_BYTES)
        return fail(MTB_INVALID_ARG, "noalloc: this structure needs %zu bytes of scratch, more "
                    "than the %zu-byte array (reduce ring_slots or the sampled region)",
                    fixed + per_chunk(1), (size_t)MTB_NOALLOC_SCRATCH_BYTES);
    // set-up, once per device: the array's device address and kernel attributes
    int dev = 0;
    MTB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NA_MAX_DEV) return fail(MTB_UNSUPPORTED, "noalloc: device ordinal %d", dev);
    std::unique_lock<std::mutex> setup_lock(g_noalloc_mu);
    if (!g_noalloc_dev[dev]) {
        void *p = nullptr;
        MTB_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        MTB_CUDA_TRY(cudaFuncSetAttribute(k_yee2d_tm<false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem_tm()));
        MTB_CUDA_TRY(cudaFuncSetAttribute(k_yee2d_tm<true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem_tm()));
        MTB_CUDA_TRY(cudaFuncSetAttribute(k_yee2d_te, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem_te()));
        MTB_CUDA_TRY(cudaFuncSetAttribute(k_dft_contract,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)(sizeof(float2) * 64 * 256)));
        g_noalloc_dev[dev] = static_cast<unsigned char *>(p);
    }
    unsigned char *base = g_noalloc_dev[dev];
    setup_lock.unlock();
    size_t off = 0;
    auto take = [&](size_t bytes) { unsigned char *q = base + off; off += na_align(bytes); return q; };
    mtb_yee2d_struct *dS = reinterpret_cast<mtb_yee2d_struct *>(take(sizeof(mtb_yee2d_struct)));
    int *dErr = reinterpret_cast<int *>(take(256));
    mtb_dft_region *dReg = reinterpret_cast<mtb_dft_region *>(
        take(sizeof(mtb_dft_region) * (n_regions + 1)));
    int64_t *dBs = reinterpret_cast<int64_t *>(take(sizeof(int64_t) * (n_regions + 1)));
    int *dGnf = reinterpret_cast<int *>(take(sizeof(double) * (NA_MAX_GROUPS + 1)));
    int *dGoff = reinterpret_cast<int *>(take(sizeof(double) * (NA_MAX_GROUPS + 1)));
    int *dGmode = reinterpret_cast<int *>(take(sizeof(double) * (NA_MAX_GROUPS + 1)));
    double *dGdt = reinterpret_cast<double *>(take(sizeof(double) * (NA_MAX_GROUPS + 1)));
    double *dFreq = reinterpret_cast<double *>(take(sizeof(double) * (total_nf + 1)));
    int *dBlk = reinterpret_cast<int *>(take(sizeof(int) * (n_blocks + 1)));
    int4 *dWork = reinterpret_cast<int4 *>(take(sizeof(int4) * n_work));
    float *dRing = n_regions > 0 ? reinterpret_cast<float *>(
                                       take(sizeof(float) * (size_t)ring_slots * ring_slot_elems))
                                 : nullptr;
    double *dCoef = reinterpret_cast<double *>(take(sizeof(double) * 2 * CH));
    float *dAmp = reinterpret_cast<float *>(take(sizeof(float) * 2 * CH));
    float *dPhase = reinterpret_cast<float *>(take(sizeof(float) * 4 * (size_t)CH *
                                                   std::max(total_nf, 1)));
    // descriptors in; the error flag must start at zero
    MTB_CUDA_TRY(cudaMemcpyAsync(dS, s, sizeof(mtb_yee2d_struct), cudaMemcpyHostToDevice, st));
    MTB_CUDA_TRY(cudaMemsetAsync(dErr, 0, sizeof(int), st));
    if (n_regions > 0) {
        MTB_CUDA_TRY(cudaMemcpyAsync(dReg, regions, sizeof(mtb_dft_region) * n_regions,
                                     cudaMemcpyHostToDevice, st));
        MTB_CUDA_TRY(cudaMemcpyAsync(dBs, bs, sizeof(int64_t) * (n_regions + 1),
                                     cudaMemcpyHostToDevice, st));
        MTB_CUDA_TRY(cudaMemcpyAsync(dGnf, gnf, sizeof(int) * (n_groups + 1),
                                     cudaMemcpyHostToDevice, st));
        MTB_CUDA_TRY(cudaMemcpyAsync(dGoff, goff, sizeof(int) * (n_groups + 1),
                                     cudaMemcpyHostToDevice, st));
        MTB_CUDA_TRY(cudaMemcpyAsync(dGmode, gmode, sizeof(int) * (n_groups + 1),
                                     cudaMemcpyHostToDevice, st));
        MTB_CUDA_TRY(cudaMemcpyAsync(dGdt, gdt, sizeof(double) * (n_groups + 1),
                                     cudaMemcpyHostToDevice, st));
        for (int g = 0; g < n_groups; ++g)
            MTB_CUDA_TRY(cudaMemcpyAsync(dFreq + goff[g], groups[g].freqs,
                                         sizeof(double) * gnf[g], cudaMemcpyHostToDevice, st));
    }
    k_na_struct<<<1, 256, 0, st>>>(dS, dErr, ring_slot_elems);
    MTB_CHECK_LAUNCH();
    // the checks' verdict before any step kernel: a rejected call leaves the
    // caller's fields, CPML memory and accumulators untouched
    int flag = 0;
    MTB_CUDA_TRY(cudaMemcpyAsync(&flag, dErr, sizeof(int), cudaMemcpyDeviceToHost, st));
    MTB_CUDA_TRY(cudaStreamSynchronize(st));
    if (flag & NA_ERR_ROWS)
        return fail(MTB_INVALID_ARG, "noalloc: a source row_ptr does not start at 0, end at n "
                    "and never decrease");
    if (flag & NA_ERR_LINES) return fail(MTB_INVALID_ARG, "noalloc: a line sample is out of range");
    if (flag & NA_ERR_COLS)
        return fail(MTB_INVALID_ARG, "noalloc: source columns are not in ascending order within "
                    "a row");
    k_na_work<<<(n_work + 255) / 256, 256, 0, st>>>(dWork, S.nx, rows, nch, n_work);
    MTB_CHECK_LAUNCH();
    if (n_blocks > 0) {
        k_na_blk<<<(unsigned)((n_blocks + 255) / 256), 256, 0, st>>>(dBlk, dBs, n_regions,
                                                                     n_blocks);
        MTB_CHECK_LAUNCH();
    }
    const int blocks = (n_work + WARPS2D - 1) / WARPS2D;
    int par = parity;
    bool first = true;
    for (int c0 = 0; c0 < k; c0 += CH) {
        const int n = std::min(CH, k - c0);
        if (coef_e)
            MTB_CUDA_TRY(cudaMemcpyAsync(dCoef, coef_e + c0, sizeof(double) * n,
                                         cudaMemcpyHostToDevice, st));
        if (coef_h)
            MTB_CUDA_TRY(cudaMemcpyAsync(dCoef + n, coef_h + c0, sizeof(double) * n,
                                         cudaMemcpyHostToDevice, st));
        k_na_amp<<<(n + 255) / 256, 256, 0, st>>>(dAmp, dCoef, n, coef_e != nullptr,
                                                  coef_h != nullptr);
        MTB_CHECK_LAUNCH();
        if (n_regions > 0) {
            const int64_t ne = (int64_t)n * total_nf;
            k_na_phase<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(
                dPhase, dFreq, dGnf, dGoff, dGdt, dGmode, n_groups, total_nf, t0 + c0, n);
            MTB_CHECK_LAUNCH();
        }
        int slot = 0;
        for (int q = 0; q < n; ++q) {
            Ctx2D C;
            C.amp_e = dAmp + q;
            C.amp_h = dAmp + n + q;
            C.ring = dRing ? dRing + (size_t)slot * ring_slot_elems : nullptr;
            C.err = dErr;
            C.par = par;
            C.first = first ? 1 : 0;
            C.wr = 1;                              // unused by the row-march kernels
            C.pst = 0;
            if (S.pol == MTB_TM) {
                if (first)
                    k_yee2d_tm<true><<<blocks, 32 * WARPS2D, smem_tm(), st>>>(dS, dWork, n_work, C);
                else
                    k_yee2d_tm<false><<<blocks, 32 * WARPS2D, smem_tm(), st>>>(dS, dWork, n_work, C);
            } else {
                k_yee2d_te<<<blocks, 32 * WARPS2D, smem_te(), st>>>(dS, dWork, n_work, C);
            }
            MTB_CHECK_LAUNCH();
            par ^= 1;
            first = false;
            ++slot;
            if ((slot == ring_slots || q == n - 1) && n_regions > 0 && n_blocks > 0) {
                k_dft_contract<<<(unsigned)n_blocks, NA_CT, sizeof(float2) * slot * maxnf, st>>>(
                    dReg, dBlk, dBs, dGnf, dGoff, total_nf, dPhase, q + 1 - slot, slot, dRing,
                    ring_slot_elems);
                MTB_CHECK_LAUNCH();
                slot = 0;
            } else if (slot == ring_slots || q == n - 1) {
                slot = 0;
            }
        }
    }
    MTB_CUDA_TRY(cudaMemcpyAsync(&flag, dErr, sizeof(int), cudaMemcpyDeviceToHost, st));
    MTB_CUDA_TRY(cudaStreamSynchronize(st));
    if (flag)
        return fail(MTB_DEVICE_TIMEOUT, "noalloc: a bounded wait for a staged row copy expired");
    return MTB_OK;
}
