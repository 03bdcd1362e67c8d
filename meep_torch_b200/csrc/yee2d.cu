// Batched 2D Yee step (TM and TE) for sm_100a.
//
// One warp marches down rows i0..i1-1 of a 128-column strip of one
// structure: lane L owns columns c0+4L .. c0+4L+3 (one float4 per array and
// row). Each iteration fuses the reference's whole step for one row:
//   TM (core/stepper_tm.py:234-254): H(n+1/2) of row i from Ez(n) of rows
//      i, i+1 -> magnetic sheet source -> Dz(n+1) of row i from H rows
//      i-1, i -> electric source -> Ez = Dz / eps.
//   TE (core/stepper_te.py:178-190): D/E(n+1/2) of row i+1 from Hz(n) rows
//      i, i+1 -> source into Dy -> E = D / eps -> Hz(n+1) of row i.
// Ez (TM) and Ex/Ey (TE) are not stored: they are D / eps, recomputed where
// needed, so the per-cell traffic is read+write of the three stored fields
// plus one (TM) or two (TE) eps reads. Halo values (the row above the strip,
// the columns left/right of it) are recomputed from the neighbours' old
// values, which is why every evolving array is a ping-pong pair.
// CPML memory is only touched where its profile is active (a != 0 or
// b != 1); outside the layers it is identically zero, as in the reference.
#include <algorithm>
#include <vector>

#include "mtb_common.cuh"

namespace mtb {

constexpr int MAXL = 16;          // line samples per structure
constexpr int WARPS2D = 4;        // warps per block

struct Ctx2D {
    const float *amp_e;           // coefficient row of this step [n_cols]
    const float *amp_h;
    float *ring;                  // ring slot of this step
    int par;                      // buffer holding the old state
    int first;                    // first step executed by the plan
};

__device__ __forceinline__ void ld4(const float *p, float (&v)[4]) {
    const float4 x = *reinterpret_cast<const float4 *>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void ldg4(const float *p, float (&v)[4]) {
    const float4 x = __ldg(reinterpret_cast<const float4 *>(p));
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void st4(float *p, const float (&v)[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void zero4(float (&v)[4]) { v[0] = v[1] = v[2] = v[3] = 0.f; }
__device__ __forceinline__ void copy4(float (&d)[4], const float (&s)[4]) {
    d[0] = s[0]; d[1] = s[1]; d[2] = s[2]; d[3] = s[3];
}

// F[row, jb+q] -= amp * w for the cells of `row` in `cl` (CSR by row).
__device__ __forceinline__ void apply_cells(const mtb_cells &cl, int row, const float *amp,
                                            int jb, float (&v)[4]) {
    if (cl.n == 0) return;
    const int e0 = __ldg(cl.row_ptr + row), e1 = __ldg(cl.row_ptr + row + 1);
    if (e0 == e1) return;
    const float a = __ldg(amp + cl.amp_col);
    for (int e = e0; e < e1; ++e) {
        const int c = __ldg(cl.col + e) - jb;
        const float w = __ldg(cl.w + e);
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (c == q) v[q] -= a * w;
    }
}
// scalar variant for a halo cell (row, col)
__device__ __forceinline__ float apply_cell1(const mtb_cells &cl, int row, int col,
                                             const float *amp, float v) {
    if (cl.n == 0) return v;
    const int e0 = __ldg(cl.row_ptr + row), e1 = __ldg(cl.row_ptr + row + 1);
    if (e0 == e1) return v;
    const float a = __ldg(amp + cl.amp_col);
    for (int e = e0; e < e1; ++e)
        if (__ldg(cl.col + e) == col) v -= a * __ldg(cl.w + e);
    return v;
}

// Copy this row's values of component `comp` into the line samples.
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

template <bool EXPL>
__device__ __forceinline__ void tm_warp(const mtb_yee2d_struct &S, const int i0, const int i1,
                                        const int c0, const Ctx2D &C,
                                        const mtb_line_sample *L, const int nl) {
    const int lane = threadIdx.x & 31;
    const int nx = S.nx, ny = S.ny;
    const int64_t P = S.pitch;
    const int jb = c0 + 4 * lane;
    const bool act = jb < S.pitch;
    const float dt = S.dt;
    const float rdx = 1.0f / S.dx;
    const int par = C.par;
    const float *__restrict__ Dz = S.f_main[par];
    float *__restrict__ Dzn = S.f_main[par ^ 1];
    const float *__restrict__ Hx = S.f_x[par];
    float *__restrict__ Hxn = S.f_x[par ^ 1];
    const float *__restrict__ Hy = S.f_y[par];
    float *__restrict__ Hyn = S.f_y[par ^ 1];
    const float *__restrict__ eps = S.eps_a;
    const float *__restrict__ Eex = S.e_explicit;
    const float *__restrict__ pEzy = S.psi[0][par];
    float *__restrict__ pEzyN = S.psi[0][par ^ 1];
    const float *__restrict__ pEzx = S.psi[1][par];
    float *__restrict__ pEzxN = S.psi[1][par ^ 1];
    const float *__restrict__ pHyx = S.psi[2][par];
    float *__restrict__ pHyxN = S.psi[2][par ^ 1];
    const float *__restrict__ pHxy = S.psi[3][par];
    float *__restrict__ pHxyN = S.psi[3][par ^ 1];
    const bool pmc = S.y_pmc != 0;
    float *ring = C.ring;

    // lane-constant column data
    bool vC[4], vHx[4], vDz[4], hyA[4], eyA[4];
    float hyb[4], hya[4], eyb[4], eya[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        vC[q] = j < ny;
        vHx[q] = j <= ny - 2;
        vDz[q] = pmc ? (j < ny) : (j >= 1 && j <= ny - 2);
        hyb[q] = vHx[q] ? __ldg(S.hy_b + j) : 1.f;
        hya[q] = vHx[q] ? __ldg(S.hy_a + j) : 0.f;
        eyb[q] = vC[q] ? __ldg(S.ey_b + j) : 1.f;
        eya[q] = vC[q] ? __ldg(S.ey_a + j) : 0.f;
        hyA[q] = vHx[q] && (hya[q] != 0.f || hyb[q] != 1.f);
        eyA[q] = vDz[q] && (eya[q] != 0.f || eyb[q] != 1.f);
    }
    const bool anyHy = act && (hyA[0] || hyA[1] || hyA[2] || hyA[3]);
    const bool anyEy = act && (eyA[0] || eyA[1] || eyA[2] || eyA[3]);
    // left halo column (lane 0): Hx(i, c0-1)
    const int jl = c0 - 1;
    const bool hasL = (lane == 0) && jl >= 0 && jl <= ny - 2;
    float hybL = 1.f, hyaL = 0.f;
    if (hasL) { hybL = __ldg(S.hy_b + jl); hyaL = __ldg(S.hy_a + jl); }
    const bool hyAL = hasL && (hyaL != 0.f || hybL != 1.f);
    const int jr = c0 + 128;   // right halo column (lane 31): Ez(i, c0+128)

    auto ezrow = [&](int i, float (&dz)[4], float (&ep)[4], float (&ez)[4]) {
        if (act && i >= 0 && i < nx) {
            ld4(Dz + i * P + jb, dz);
            ldg4(eps + i * P + jb, ep);
            if (EXPL) {
                ldg4(Eex + i * P + jb, ez);
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) ez[q] = vC[q] ? dz[q] / ep[q] : 0.f;
            }
        } else {
            zero4(dz); zero4(ez);
            ep[0] = ep[1] = ep[2] = ep[3] = 1.f;
        }
    };
    auto ezat = [&](int i, int j) -> float {
        if (i < 0 || i >= nx || j < 0 || j >= ny) return 0.f;
        if (EXPL) return __ldg(Eex + i * P + j);
        return Dz[i * P + j] / __ldg(eps + i * P + j);
    };
    // Hy(n+1/2) of row i from Ez rows i (ea) and i+1 (eb) (core/stepper_tm.py:97-100, :119-128)
    auto hy_new = [&](int i, const float (&ea)[4], const float (&eb)[4], float (&out)[4],
                      bool own) {
        if (!(act && i >= 0 && i < nx)) { zero4(out); return; }
        ld4(Hy + i * P + jb, out);
        if (i > nx - 2) return;                       // padding row of the box
        const float b = __ldg(S.hx_b + i), a = __ldg(S.hx_a + i);
        const bool pa = (a != 0.f) || (b != 1.f);
        float ps[4];
        if (pa) ld4(pEzx + i * P + jb, ps); else zero4(ps);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (!vC[q]) continue;
            const float d = (eb[q] - ea[q]) * rdx;
            float c = d;
            if (pa) { ps[q] = b * ps[q] + a * d; c = d + ps[q]; }
            out[q] = out[q] + dt * c;
        }
        if (pa && own) st4(pEzxN + i * P + jb, ps);
        apply_cells(S.src_h1, i, C.amp_h, jb, out);
    };

    // ---- prologue: Ez rows i0-1 and i0, Hy(n+1/2) of row i0-1 (halo)
    float dzB[4], epB[4], ezB[4], hyP[4];
    {
        float dA[4], eA[4], zA[4];
        ezrow(i0 - 1, dA, eA, zA);
        ezrow(i0, dzB, epB, ezB);
        if (i0 >= 1) hy_new(i0 - 1, zA, ezB, hyP, false); else zero4(hyP);
    }
    float ezLB = (lane == 0) ? ezat(i0, jl) : 0.f;
    float ezRB = (lane == 31) ? ezat(i0, jr) : 0.f;

    for (int i = i0; i < i1; ++i) {
        float dzC[4], epC[4], ezC[4];
        ezrow(i + 1, dzC, epC, ezC);
        const float ezLC = (lane == 0) ? ezat(i + 1, jl) : 0.f;
        const float ezRC = (lane == 31) ? ezat(i + 1, jr) : 0.f;
        const int64_t ro = i * P + jb;

        // Hy(n+1/2), row i
        float hyN[4];
        hy_new(i, ezB, ezC, hyN, true);

        // Hx(n+1/2), row i (core/stepper_tm.py:91-94, :121-128)
        float hxN[4];
        {
            float ezr = __shfl_down_sync(0xffffffffu, ezB[0], 1);
            if (lane == 31) ezr = ezRB;
            if (act) ld4(Hx + ro, hxN); else zero4(hxN);
            float ps[4];
            if (anyHy) ld4(pEzy + ro, ps); else zero4(ps);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (!vHx[q]) continue;
                const float er = (q < 3) ? ezB[q + 1] : ezr;
                const float d = (er - ezB[q]) * rdx;
                float c = d;
                if (hyA[q]) { ps[q] = hyb[q] * ps[q] + hya[q] * d; c = d + ps[q]; }
                hxN[q] = hxN[q] - dt * c;
            }
            if (anyHy) st4(pEzyN + ro, ps);
            if (act) apply_cells(S.src_h2, i, C.amp_h, jb, hxN);
        }
        // left neighbour Hx(n+1/2)(i, j-1)
        float hxl0 = __shfl_up_sync(0xffffffffu, hxN[3], 1);
        if (lane == 0) {
            float v = 0.f;
            if (hasL) {
                const float d = (ezB[0] - ezLB) * rdx;
                float c = d;
                if (hyAL) c = d + (hybL * pEzy[i * P + jl] + hyaL * d);
                v = Hx[i * P + jl] - dt * c;
                v = apply_cell1(S.src_h2, i, jl, C.amp_h, v);
            }
            hxl0 = v;
        }

        // Dz(n+1), row i (core/stepper_tm.py:136-166), then source and E
        float dzN[4], ezN[4];
        {
            const bool irow = (i >= 1 && i <= nx - 2);
            float bx = 1.f, ax = 0.f;
            if (irow) { bx = __ldg(S.ex_b + i); ax = __ldg(S.ex_a + i); }
            const bool pxA = act && irow && (ax != 0.f || bx != 1.f);
            const bool pyA = irow && anyEy;
            float px[4], py[4];
            if (pxA) ld4(pHyx + ro, px); else zero4(px);
            if (pyA) ld4(pHxy + ro, py); else zero4(py);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float dz = dzB[q];
                if (irow && vDz[q]) {
                    const float hxm = (q == 0) ? hxl0 : hxN[q - 1];
                    const float dhy = (hyN[q] - hyP[q]) * rdx;
                    const float dhx = (hxN[q] - hxm) * rdx;
                    float p1 = 0.f, p2 = 0.f;
                    if (pxA) { p1 = bx * px[q] + ax * dhy; px[q] = p1; }
                    if (eyA[q]) { p2 = eyb[q] * py[q] + eya[q] * dhx; py[q] = p2; }
                    const float curl = ((dhy + p1) - dhx) - p2;
                    dz = dz + dt * curl;
                }
                dzN[q] = dz;
            }
            if (pxA) st4(pHyxN + ro, px);
            if (pyA) st4(pHxyN + ro, py);
            if (act) apply_cells(S.src_e, i, C.amp_e, jb, dzN);
#pragma unroll
            for (int q = 0; q < 4; ++q) ezN[q] = vC[q] ? dzN[q] / epB[q] : 0.f;
        }
        if (act) {
            st4(Hxn + ro, hxN);
            st4(Hyn + ro, hyN);
            st4(Dzn + ro, dzN);
            if (S.ring_full[0] >= 0) st4(ring + S.ring_full[0] + ro, ezN);
            if (S.ring_full[1] >= 0) st4(ring + S.ring_full[1] + ro, hxN);
            if (S.ring_full[2] >= 0) st4(ring + S.ring_full[2] + ro, hyN);
        }
        if (nl) {
            sample_row(L, nl, MTB_C2_MAIN, i, jb, act, ezN, ring);
            sample_row(L, nl, MTB_C2_X, i, jb, act, hxN, ring);
            sample_row(L, nl, MTB_C2_Y, i, jb, act, hyN, ring);
        }
        copy4(hyP, hyN);
        copy4(dzB, dzC);
        copy4(epB, epC);
        copy4(ezB, ezC);
        ezLB = ezLC;
        ezRB = ezRC;
    }
}

// ------------------------------------------------------------------ TE

__device__ __forceinline__ void te_warp(const mtb_yee2d_struct &S, const int i0, const int i1,
                                        const int c0, const Ctx2D &C,
                                        const mtb_line_sample *L, const int nl) {
    const int lane = threadIdx.x & 31;
    const int nx = S.nx, ny = S.ny;
    const int64_t P = S.pitch;
    const int jb = c0 + 4 * lane;
    const bool act = jb < S.pitch;
    const float dt = S.dt;
    const float rdx = 1.0f / S.dx;
    const int par = C.par;
    const float *__restrict__ Hz = S.f_main[par];
    float *__restrict__ Hzn = S.f_main[par ^ 1];
    const float *__restrict__ Dx = S.f_x[par];
    float *__restrict__ Dxn = S.f_x[par ^ 1];
    const float *__restrict__ Dy = S.f_y[par];
    float *__restrict__ Dyn = S.f_y[par ^ 1];
    const float *__restrict__ epx = S.eps_a;
    const float *__restrict__ epy = S.eps_b;
    const float *__restrict__ pHzy = S.psi[0][par];
    float *__restrict__ pHzyN = S.psi[0][par ^ 1];
    const float *__restrict__ pHzx = S.psi[1][par];
    float *__restrict__ pHzxN = S.psi[1][par ^ 1];
    const float *__restrict__ pEyx = S.psi[2][par];
    float *__restrict__ pEyxN = S.psi[2][par ^ 1];
    const float *__restrict__ pExy = S.psi[3][par];
    float *__restrict__ pExyN = S.psi[3][par ^ 1];
    float *ring = C.ring;

    bool vHz[4], vEx[4], vDxU[4], vEy[4], eyA[4], hyA[4];
    float eyb[4], eya[4], hyb[4], hya[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        vHz[q] = j <= ny - 2;
        vEx[q] = j < ny;
        vDxU[q] = j >= 1 && j <= ny - 2;
        vEy[q] = j <= ny - 2;
        eyb[q] = vEx[q] ? __ldg(S.ey_b + j) : 1.f;
        eya[q] = vEx[q] ? __ldg(S.ey_a + j) : 0.f;
        hyb[q] = vHz[q] ? __ldg(S.hy_b + j) : 1.f;
        hya[q] = vHz[q] ? __ldg(S.hy_a + j) : 0.f;
        eyA[q] = vDxU[q] && (eya[q] != 0.f || eyb[q] != 1.f);
        hyA[q] = vHz[q] && (hya[q] != 0.f || hyb[q] != 1.f);
    }
    const bool anyEy = act && (eyA[0] || eyA[1] || eyA[2] || eyA[3]);
    const bool anyHy = act && (hyA[0] || hyA[1] || hyA[2] || hyA[3]);
    const int jl = c0 - 1;          // left halo: Hz(r, c0-1)
    const int jr = c0 + 128;        // right halo: Ex(n+1/2)(r, c0+128)
    const bool hasR = (lane == 31) && jr <= ny - 1;
    float eybR = 1.f, eyaR = 0.f;
    const bool updR = hasR && jr >= 1 && jr <= ny - 2;
    if (updR) { eybR = __ldg(S.ey_b + jr); eyaR = __ldg(S.ey_a + jr); }
    const bool eyAR = updR && (eyaR != 0.f || eybR != 1.f);

    auto hzrow = [&](int r, float (&v)[4]) {
        if (act && r >= 0 && r < nx) ld4(Hz + r * P + jb, v); else zero4(v);
    };
    auto hzat = [&](int r, int j) -> float {
        if (r < 0 || r > nx - 2 || j < 0 || j > ny - 2) return 0.f;
        return Hz[r * P + j];
    };

    // D/E(n+1/2) of row r from Hz(n) rows r-1 (hp) and r (hc)
    // (core/stepper_te.py:79-111 D update, :120-134 source, :150-175 E)
    auto e_row = [&](int r, const float (&hp)[4], const float (&hc)[4], float hzL, float hzR,
                     bool own, float (&ex)[4], float (&ey)[4], float &exR) {
        exR = 0.f;
        if (r < 0 || r >= nx) { zero4(ex); zero4(ey); return; }
        const int64_t ro = r * P + jb;
        // Dx, row r (valid rows 0..nx-2)
        float dxN[4];
        if (act) ld4(Dx + ro, dxN); else zero4(dxN);
        float hl = __shfl_up_sync(0xffffffffu, hc[3], 1);
        if (lane == 0) hl = hzL;
        if (r <= nx - 2) {
            float py[4];
            if (anyEy) ld4(pHzy + ro, py); else zero4(py);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (!vDxU[q]) continue;
                const float hm = (q == 0) ? hl : hc[q - 1];
                const float d = (hc[q] - hm) * rdx;
                float c = d;
                if (eyA[q]) { py[q] = eyb[q] * py[q] + eya[q] * d; c = d + py[q]; }
                dxN[q] = dxN[q] + dt * c;
            }
            if (anyEy && own) st4(pHzyN + ro, py);
            float ep[4];
            if (act) ldg4(epx + ro, ep); else ep[0] = ep[1] = ep[2] = ep[3] = 1.f;
#pragma unroll
            for (int q = 0; q < 4; ++q) ex[q] = vEx[q] ? dxN[q] / ep[q] : 0.f;
            if (hasR) {
                float dxr = Dx[r * P + jr];
                if (updR) {
                    const float d = (hzR - hc[3]) * rdx;
                    float c = d;
                    if (eyAR) c = d + (eybR * pHzy[r * P + jr] + eyaR * d);
                    dxr = dxr + dt * c;
                }
                exR = dxr / __ldg(epx + r * P + jr);
            }
        } else {
            zero4(ex);
        }
        // Dy, row r (valid rows 0..nx-1; updated 1..nx-2)
        float dyN[4];
        if (act) ld4(Dy + ro, dyN); else zero4(dyN);
        const bool irow = r >= 1 && r <= nx - 2;
        float bx = 1.f, ax = 0.f;
        if (irow) { bx = __ldg(S.ex_b + r); ax = __ldg(S.ex_a + r); }
        const bool pxA = act && irow && (ax != 0.f || bx != 1.f);
        float px[4];
        if (pxA) ld4(pHzx + ro, px); else zero4(px);
        if (irow) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (!vEy[q]) continue;
                const float d = (hc[q] - hp[q]) * rdx;
                float c = d;
                if (pxA) { px[q] = bx * px[q] + ax * d; c = d + px[q]; }
                dyN[q] = dyN[q] - dt * c;
            }
        }
        if (pxA && own) st4(pHzxN + ro, px);
        if (act) apply_cells(S.src_e, r, C.amp_e, jb, dyN);
        float ep[4];
        if (act) ldg4(epy + ro, ep); else ep[0] = ep[1] = ep[2] = ep[3] = 1.f;
#pragma unroll
        for (int q = 0; q < 4; ++q) ey[q] = vEy[q] ? dyN[q] / ep[q] : 0.f;
        if (own && act) {
            st4(Dxn + ro, dxN);
            st4(Dyn + ro, dyN);
            if (S.ring_full[1] >= 0) st4(ring + S.ring_full[1] + ro, ex);
            if (S.ring_full[2] >= 0) st4(ring + S.ring_full[2] + ro, ey);
        }
        if (own && nl) {
            sample_row(L, nl, MTB_C2_X, r, jb, act, ex, ring);
            sample_row(L, nl, MTB_C2_Y, r, jb, act, ey, ring);
        }
    };

    // ---- prologue
    float hzA[4], hzB[4], exB[4], eyB[4], exRB;
    hzrow(i0 - 1, hzA);
    hzrow(i0, hzB);
    float hzLB = (lane == 0) ? hzat(i0, jl) : 0.f;
    float hzRB = (lane == 31) ? hzat(i0, jr) : 0.f;
    e_row(i0, hzA, hzB, hzLB, hzRB, true, exB, eyB, exRB);

    for (int i = i0; i < i1; ++i) {
        float hzC[4], exC[4], eyC[4], exRC;
        hzrow(i + 1, hzC);
        const float hzLC = (lane == 0) ? hzat(i + 1, jl) : 0.f;
        const float hzRC = (lane == 31) ? hzat(i + 1, jr) : 0.f;
        e_row(i + 1, hzB, hzC, hzLC, hzRC, i + 1 < i1, exC, eyC, exRC);

        // Hz(n+1), row i (core/stepper_te.py:113-117)
        const int64_t ro = i * P + jb;
        float hzN[4];
        copy4(hzN, hzB);
        if (i <= nx - 2) {
            const float bx = __ldg(S.hx_b + i), ax = __ldg(S.hx_a + i);
            const bool pxA = act && (ax != 0.f || bx != 1.f);
            float p1v[4], p2v[4];
            if (pxA) ld4(pEyx + ro, p1v); else zero4(p1v);
            if (anyHy) ld4(pExy + ro, p2v); else zero4(p2v);
            float exr = __shfl_down_sync(0xffffffffu, exB[0], 1);
            if (lane == 31) exr = exRB;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (!vHz[q]) continue;
                const float exn = (q < 3) ? exB[q + 1] : exr;
                const float dey = (eyC[q] - eyB[q]) * rdx;
                const float dex = (exn - exB[q]) * rdx;
                float p1 = 0.f, p2 = 0.f;
                if (pxA) { p1 = bx * p1v[q] + ax * dey; p1v[q] = p1; }
                if (hyA[q]) { p2 = hyb[q] * p2v[q] + hya[q] * dex; p2v[q] = p2; }
                const float curl = ((dey + p1) - dex) - p2;
                hzN[q] = hzN[q] - dt * curl;
            }
            if (pxA) st4(pEyxN + ro, p1v);
            if (anyHy) st4(pExyN + ro, p2v);
            if (act) apply_cells(S.src_h1, i, C.amp_h, jb, hzN);
        }
        if (act) {
            st4(Hzn + ro, hzN);
            if (S.ring_full[0] >= 0) st4(ring + S.ring_full[0] + ro, hzN);
        }
        if (nl) sample_row(L, nl, MTB_C2_MAIN, i, jb, act, hzN, ring);
        copy4(hzB, hzC);
        copy4(exB, exC);
        copy4(eyB, eyC);
        exRB = exRC;
    }
}

__global__ void __launch_bounds__(32 * WARPS2D) k_yee2d_step(
    const mtb_yee2d_struct *__restrict__ SS, const int4 *__restrict__ work, int n_work,
    Ctx2D C) {
    __shared__ mtb_line_sample sl[WARPS2D][MAXL];
    const int wib = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int wid = blockIdx.x * WARPS2D + wib;
    if (wid >= n_work) return;
    const int4 w = work[wid];
    const mtb_yee2d_struct &S = SS[w.x];
    const int nl = S.n_lines;
    if (lane < nl) sl[wib][lane] = S.lines[lane];
    __syncwarp();
    if (S.pol == MTB_TM) {
        if (C.first && S.explicit_e)
            tm_warp<true>(S, w.y, w.z, w.w, C, sl[wib], nl);
        else
            tm_warp<false>(S, w.y, w.z, w.w, C, sl[wib], nl);
    } else {
        te_warp(S, w.y, w.z, w.w, C, sl[wib], nl);
    }
}

}  // namespace mtb

using namespace mtb;

struct mtb_yee2d_plan {
    int n_structs = 0;
    DevBuf structs_d, work_d, amp_d;
    HostBuf amp_h;
    int n_work = 0;
    int n_cols = 0;
    int rows = 32;
    int par = 0;
    int first = 1;
    int64_t last_launches = 0;
    DftState dft;
    LaunchTimer timer;
};

static int check_ptr(const void *p, const char *what, int s) {
    if (!p) return fail(MTB_INVALID_ARG, "structure %d: %s is null", s, what);
    if (reinterpret_cast<uintptr_t>(p) & 15)
        return fail(MTB_INVALID_ARG, "structure %d: %s is not 16-byte aligned", s, what);
    return MTB_OK;
}

extern "C" {

int mtb_yee2d_plan_create(const mtb_yee2d_struct *structs, int32_t n, const mtb_dft_region *regions,
                          int32_t n_regions, const mtb_phase_group *groups, int32_t n_groups,
                          int64_t ring_slot_elems, int32_t n_amp_cols, const mtb_tuning *tuning,
                          mtb_yee2d_plan **out) {
    if (!out) return fail(MTB_INVALID_ARG, "out is null");
    *out = nullptr;
    if (n < 1 || !structs) return fail(MTB_INVALID_ARG, "need at least one structure");
    if (n_amp_cols < 0) return fail(MTB_INVALID_ARG, "n_amp_cols < 0");
    int rows = (tuning && tuning->rows_per_warp > 0) ? tuning->rows_per_warp : 32;
    int slots = (tuning && tuning->ring_slots > 0) ? tuning->ring_slots : 16;
    if (ring_slot_elems < 0 || (ring_slot_elems & 3))
        return fail(MTB_INVALID_ARG, "ring_slot_elems must be a non-negative multiple of 4");
    int64_t n_work = 0;
    for (int s = 0; s < n; ++s) {
        const mtb_yee2d_struct &S = structs[s];
        if (S.pol != MTB_TM && S.pol != MTB_TE)
            return fail(MTB_INVALID_ARG, "structure %d: pol must be MTB_TM or MTB_TE", s);
        if (S.nx < 3 || S.ny < 3)
            return fail(MTB_INVALID_ARG, "structure %d: nx, ny must be >= 3 (got %d, %d)", s, S.nx,
                        S.ny);
        if (S.pitch < S.ny || (S.pitch & 3))
            return fail(MTB_INVALID_ARG, "structure %d: pitch %d must be >= ny and a multiple of 4",
                        s, S.pitch);
        if (!(S.dt > 0.f) || !(S.dx > 0.f))
            return fail(MTB_INVALID_ARG, "structure %d: dt, dx must be > 0", s);
        if (S.pol == MTB_TE && S.y_pmc)
            return fail(MTB_UNSUPPORTED, "structure %d: y_pmc is a TM option", s);
        int rc;
        for (int b = 0; b < 2; ++b) {
            if ((rc = check_ptr(S.f_main[b], "f_main", s))) return rc;
            if ((rc = check_ptr(S.f_x[b], "f_x", s))) return rc;
            if ((rc = check_ptr(S.f_y[b], "f_y", s))) return rc;
            for (int k = 0; k < 4; ++k)
                if ((rc = check_ptr(S.psi[k][b], "psi", s))) return rc;
        }
        if ((rc = check_ptr(S.eps_a, "eps_a", s))) return rc;
        if (S.pol == MTB_TE && (rc = check_ptr(S.eps_b, "eps_b", s))) return rc;
        if (S.pol == MTB_TM && S.explicit_e && (rc = check_ptr(S.e_explicit, "e_explicit", s)))
            return rc;
        if (!S.hx_b || !S.hx_a || !S.hy_b || !S.hy_a || !S.ex_b || !S.ex_a || !S.ey_b || !S.ey_a)
            return fail(MTB_INVALID_ARG, "structure %d: null CPML profile", s);
        const mtb_cells *cl[3] = {&S.src_e, &S.src_h1, &S.src_h2};
        for (int c = 0; c < 3; ++c) {
            if (cl[c]->n < 0) return fail(MTB_INVALID_ARG, "structure %d: negative cell count", s);
            if (cl[c]->n > 0 && (!cl[c]->row_ptr || !cl[c]->col || !cl[c]->w ||
                                 cl[c]->amp_col < 0 || cl[c]->amp_col >= n_amp_cols))
                return fail(MTB_INVALID_ARG, "structure %d: source list %d has null arrays or "
                            "amp_col out of [0, %d)", s, c, n_amp_cols);
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
        n_work += (int64_t)((S.nx + rows - 1) / rows) * ((S.pitch + 127) / 128);
    }
    if (n_work > (1LL << 30)) return fail(MTB_INVALID_ARG, "batch too large");
    mtb_yee2d_plan *p = new mtb_yee2d_plan();
    p->n_structs = n;
    p->rows = rows;
    p->n_cols = n_amp_cols;
    p->n_work = (int)n_work;
    int rc = p->dft.init(regions, n_regions, groups, n_groups, ring_slot_elems, slots);
    if (!rc) rc = p->structs_d.ensure(sizeof(mtb_yee2d_struct) * n);
    if (!rc) rc = p->work_d.ensure(sizeof(int4) * n_work);
    if (rc) { p->dft.release(); delete p; return rc; }
    std::vector<int4> work;
    work.reserve(n_work);
    for (int s = 0; s < n; ++s)
        for (int i0 = 0; i0 < structs[s].nx; i0 += rows)
            for (int c0 = 0; c0 < structs[s].pitch; c0 += 128)
                work.push_back(make_int4(s, i0, std::min(i0 + rows, structs[s].nx), c0));
    cudaError_t e = cudaMemcpy(p->structs_d.p, structs, sizeof(mtb_yee2d_struct) * n,
                               cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(p->work_d.p, work.data(), sizeof(int4) * n_work, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        p->dft.release();
        delete p;
        return fail(MTB_CUDA_ERROR, "plan upload failed: %s", cudaGetErrorString(e));
    }
    *out = p;
    return MTB_OK;
}

int mtb_yee2d_run(mtb_yee2d_plan *p, int64_t t0, int32_t k, const double *coef_e,
                  const double *coef_h, void *stream) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    if (k < 0) return fail(MTB_INVALID_ARG, "k < 0");
    p->last_launches = 0;
    if (k == 0) return MTB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const int nc = std::max(p->n_cols, 1);
    const size_t per = (size_t)k * nc;
    int rc;
    if ((rc = p->amp_h.ensure(2 * per * sizeof(float)))) return rc;
    if ((rc = p->amp_d.ensure(2 * per * sizeof(float)))) return rc;
    if ((rc = p->dft.upload_phases(t0, k, st))) return rc;   // syncs the stream first
    float *ah = p->amp_h.as<float>();
    for (size_t i = 0; i < per; ++i) {
        ah[i] = coef_e ? (float)coef_e[i] : 0.f;
        ah[per + i] = coef_h ? (float)coef_h[i] : 0.f;
    }
    MTB_CUDA_TRY(cudaMemcpyAsync(p->amp_d.p, p->amp_h.p, 2 * per * sizeof(float),
                                 cudaMemcpyHostToDevice, st));
    const float *ad = p->amp_d.as<float>();
    const int blocks = (p->n_work + WARPS2D - 1) / WARPS2D;
    int slot = 0;
    for (int s = 0; s < k; ++s) {
        Ctx2D C;
        C.amp_e = ad + (size_t)s * nc;
        C.amp_h = ad + per + (size_t)s * nc;
        C.ring = p->dft.ring_d.as<float>() + (size_t)slot * p->dft.slot_elems;
        C.par = p->par;
        C.first = p->first;
        if ((rc = p->timer.begin(st, 0))) return rc;
        k_yee2d_step<<<blocks, 32 * WARPS2D, 0, st>>>(p->structs_d.as<mtb_yee2d_struct>(),
                                                      p->work_d.as<int4>(), p->n_work, C);
        MTB_CHECK_LAUNCH();
        if ((rc = p->timer.end(st))) return rc;
        ++p->last_launches;
        p->par ^= 1;
        p->first = 0;
        ++slot;
        if (slot == p->dft.slots || s == k - 1) {
            if (p->dft.n_regions > 0) {
                if ((rc = p->dft.contract(s + 1 - slot, slot, st, &p->timer))) return rc;
                ++p->last_launches;
            }
            slot = 0;
        }
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

int32_t mtb_yee2d_current(const mtb_yee2d_plan *p) { return p ? p->par : -1; }

int64_t mtb_yee2d_last_launches(const mtb_yee2d_plan *p) { return p ? p->last_launches : -1; }

void mtb_yee2d_plan_destroy(mtb_yee2d_plan *p) {
    if (!p) return;
    p->structs_d.release();
    p->work_d.release();
    p->amp_d.release();
    p->amp_h.release();
    p->dft.release();
    p->timer.release();
    delete p;
}

}  // extern "C"
