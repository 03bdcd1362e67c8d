// Three-pass TE step for structures whose E at a node depends on D at the
// neighbouring nodes of the other component: the in-plane tensor eps and the
// oriented (tensor) poles (core/coeffs.py:389-399, :428-456; core/stepper_te.py:
// 136-175). The one-pass TE tile recomputes E where it needs it; here E has to
// come from a two-node-wide neighbourhood of D, so E is kept in two box arrays
// (e_x, e_y: the state's own Ex, Ey) and the step runs as three launches over
// the same work items (k_te3<PASS>):
//   k_te3_d  Dx, Dy(n+1/2) from Hz(n) with their CPML memory, conductivity and
//            the soft current on Dy; the ADE poles P(n+1/2) = c1 P(n-1/2) +
//            c2 P(n-3/2) + c3 E(n-1/2) (+ c3xy * avg4(Ey(n-1/2)) on Px, c3yx *
//            avg4(Ex(n-1/2)) on Py) from the stored E;
//   k_te3_e  E(n+1/2) from rhs = D - sum P: inv_xx rhs_x + inv_xy avg4(rhs_y) on
//            Ex and inv_yy rhs_y + inv_xy avg4(rhs_x) on Ey (or rhs / eps), the
//            samples of Ex, Ey;
//   k_te3_h  Hz(n+1) from the stored E(n+1/2) with its CPML memory, magnetic
//            pairs and source, the samples of Hz.
// With chi2 / chi3 (core/stepper_te.py:160-171) pass 2 leaves the first iterate rhs / eps
// in the scratch boxes and three Jacobi sweeps (passes 3-5, before the Hz pass) end in E.
// avg4 is the reference's four-node Yee average with zero padding at the walls
// (core/stepper_te.py:52-61). Padding cells of every box stay zero.
#pragma once

namespace mtb {

// D - sum_k P_k on a float4 (o) of a box, P the stack of np planes pl floats apart
__device__ __forceinline__ void te3_rhs4(const float *D, const float *Pk, int np, uint32_t pl,
                                         uint32_t o, float (&r)[4]) {
    ld4(D + o, r);
    if (np > 0) {
        float s[4];
        pole_sum4(Pk, np, pl, o, s);
#pragma unroll
        for (int q = 0; q < 4; ++q) r[q] -= s[q];
    }
}
__device__ __forceinline__ float te3_rhs1(const float *D, const float *Pk, int np, uint32_t pl,
                                          uint32_t o) {
    float s = 0.f;
    for (int k = 0; k < np; ++k) s += Pk[k * pl + o];
    return D[o] - s;
}

// avg4 onto the Ex nodes (i, jb..jb+3) of an Ey-node array A given at rows i and
// i+1: 0.25 ((A(i, j-1) + A(i, j)) + A(i+1, j-1)) + A(i+1, j)), A(., -1) and
// A(., ny-1..) zero. a0 / a1: rows i / i+1 at jb..jb+3, l0 / l1 their column jb-1.
__device__ __forceinline__ void te3_avg_ex(const float (&a0)[4], float l0, const float (&a1)[4],
                                           float l1, int jb, int ny, float (&out)[4]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        const bool in = j <= ny - 2, inl = j >= 1 && j - 1 <= ny - 2;
        const float b0 = in ? a0[q] : 0.f, b1 = in ? a1[q] : 0.f;
        const float m0 = inl ? (q == 0 ? l0 : a0[q - 1]) : 0.f;
        const float m1 = inl ? (q == 0 ? l1 : a1[q - 1]) : 0.f;
        out[q] = 0.25f * (((m0 + b0) + m1) + b1);
    }
}

// avg4 onto the Ey nodes (i, jb..jb+3) of an Ex-node array A given at rows i-1 and
// i: 0.25 (((A(i-1, j) + A(i-1, j+1)) + A(i, j)) + A(i, j+1)), rows outside
// 0 .. nx-2 zero. p / c: rows i-1 / i at jb..jb+3, pr / cr their column jb+4.
__device__ __forceinline__ void te3_avg_ey(const float (&p)[4], float pr, const float (&c)[4],
                                           float cr, float (&out)[4]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float pn = q < 3 ? p[q + 1] : pr, cn = q < 3 ? c[q + 1] : cr;
        out[q] = 0.25f * (((p[q] + pn) + c[q]) + cn);
    }
}

// Pass 1: D(n+1/2) and the poles (one row i, columns jb .. jb+3 of a lane).
__device__ __forceinline__ void te3_d_row(const mtb_yee2d_struct &S, const int i, const int c0,
                                          const Ctx2D &C) {
    const int lane = threadIdx.x;
    const int nx = S.nx, ny = S.ny, P = S.pitch;
    const int jb = c0 + 4 * lane;
    const bool act = jb < P;
    const float dt = S.dt, rdx = 1.0f / S.dx;
    const int par = C.par, pn = par ^ 1;
    const uint32_t ro = (uint32_t)i * P + (act ? jb : P - 4);
    const float *__restrict__ Hz = S.f_main[par];
    const bool xrow = i <= nx - 2, yrow = i >= 1 && i <= nx - 2;
    const bool byE = act && xrow && band4(jb, S.yband[2], S.yband[3]);
    const bool bxE = act && yrow && in_band(i, S.xband[2], S.xband[3]);
    float hc[4], hp[4], dx[4], dy[4], p0[4], p1[4];
    zero4(hc); zero4(hp); zero4(dx); zero4(dy); zero4(p0); zero4(p1);
    float hzL = 0.f;
    if (act) {
        ld4(Hz + ro, hc);
        if (i >= 1) ld4(Hz + ro - P, hp);
        ld4(S.f_x[par] + ro, dx);
        ld4(S.f_y[par] + ro, dy);
        if (lane == 0 && jb >= 1) hzL = Hz[ro - 1];
        if (byE) ld4(S.psi[0][par] + ro, p0);
        if (bxE) ld4(S.psi[1][par] + ro, p1);
    }
    float hm0 = __shfl_up_sync(0xffffffffu, hc[3], 1);
    if (lane == 0) hm0 = hzL;
    // Dx += dt (dHz/dy + psi) on rows <= nx-2, columns 1 .. ny-2 (core/stepper_te.py:80-100)
    const bool cond = S.cond_d1[0] != nullptr;
    float c1[4] = {1.f, 1.f, 1.f, 1.f}, c2[4] = {dt, dt, dt, dt};
    if (cond && act) {
        ld4(S.cond_d1[0] + ro, c1);
        ld4(S.cond_d2[0] + ro, c2);
    }
    float dxN[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        const bool v = act && xrow && j >= 1 && j <= ny - 2;
        const bool oe = byE && j >= 1 && j <= ny - 2;
        const float eyb = oe ? __ldg(S.ey_b + j) : 1.f, eya = oe ? __ldg(S.ey_a + j) : 0.f;
        const float hm = (q == 0) ? hm0 : hc[q - 1];
        const float d = (hc[q] - hm) * rdx;
        const float pv = eyb * p0[q] + eya * d;
        const float dn = cond ? c1[q] * dx[q] + c2[q] * (d + pv) : dx[q] + dt * (d + pv);
        dxN[q] = v ? dn : (cond ? c1[q] * dx[q] : dx[q]);
        p0[q] = v ? pv : p0[q];
    }
    // Dy -= dt (dHz/dx + psi) on rows 1 .. nx-2 with the soft current
    float exb = 1.f, exa = 0.f, dyN[4];
    if (bxE) { exb = __ldg(S.ex_b + i); exa = __ldg(S.ex_a + i); }
    te_dy<true>(S, i, yrow, act, jb, exb, exa, dt, rdx, hp, hc, dy, p1, dyN, C.amp_e);
    // poles from the stored E(n-1/2)
    const uint32_t pl = (uint32_t)nx * P;
    const int npx = S.n_poles, npy = S.n_poles_y;
    if (npx > 0 && act) {
        float eo[4], ax[4];
        ld4(S.e_x + ro, eo);
        zero4(ax);
        if (S.c3xy) {
            float a0[4], a1[4], l0 = 0.f, l1 = 0.f;
            zero4(a1);
            ld4(S.e_y + ro, a0);
            if (jb >= 1) l0 = S.e_y[ro - 1];
            if (i + 1 < nx) {
                ld4(S.e_y + ro + P, a1);
                if (jb >= 1) l1 = S.e_y[ro + P - 1];
            }
            te3_avg_ex(a0, l0, a1, l1, jb, ny, ax);
        }
        const float *Pc = S.pol_p[C.pst], *Pp = S.pol_p[(C.pst + 2) % 3];
        float *Po = S.pol_p[(C.pst + 1) % 3];
#pragma unroll 1
        for (int k = 0; k < npx; ++k) {
            const uint32_t o = k * pl + ro;
            float pc[4], pp[4], k1[4], k2[4], k3[4], kx[4];
            ld4(Pc + o, pc); ld4(Pp + o, pp);
            ld4(S.pol_c[0] + o, k1); ld4(S.pol_c[1] + o, k2); ld4(S.pol_c[2] + o, k3);
            zero4(kx);
            if (S.c3xy) ld4(S.c3xy + o, kx);
#pragma unroll
            for (int q = 0; q < 4; ++q)
                pc[q] = ((k1[q] * pc[q] + k2[q] * pp[q]) + k3[q] * eo[q]) + kx[q] * ax[q];
            st4(Po + o, pc);
        }
    }
    if (npy > 0 && act) {
        float eo[4], ay[4];
        ld4(S.e_y + ro, eo);
        zero4(ay);
        if (S.c3yx) {
            float p[4], c[4], pr = 0.f, cr = 0.f;
            zero4(p); zero4(c);
            const bool hasr = jb + 4 < P;
            if (i >= 1 && i - 1 <= nx - 2) {
                ld4(S.e_x + ro - P, p);
                if (hasr) pr = S.e_x[ro - P + 4];
            }
            if (i <= nx - 2) {
                ld4(S.e_x + ro, c);
                if (hasr) cr = S.e_x[ro + 4];
            }
            te3_avg_ey(p, pr, c, cr, ay);
        }
        const float *Pc = S.pol_py[C.pst], *Pp = S.pol_py[(C.pst + 2) % 3];
        float *Po = S.pol_py[(C.pst + 1) % 3];
#pragma unroll 1
        for (int k = 0; k < npy; ++k) {
            const uint32_t o = k * pl + ro;
            float pc[4], pp[4], k1[4], k2[4], k3[4], ky[4];
            ld4(Pc + o, pc); ld4(Pp + o, pp);
            ld4(S.pol_cy[0] + o, k1); ld4(S.pol_cy[1] + o, k2); ld4(S.pol_cy[2] + o, k3);
            zero4(ky);
            if (S.c3yx) ld4(S.c3yx + o, ky);
#pragma unroll
            for (int q = 0; q < 4; ++q)
                pc[q] = ((k1[q] * pc[q] + k2[q] * pp[q]) + k3[q] * eo[q]) + ky[q] * ay[q];
            st4(Po + o, pc);
        }
    }
    if (!act) return;
    st4(S.f_x[pn] + ro, dxN);
    st4(S.f_y[pn] + ro, dyN);
    if (byE) st4(S.psi[0][pn] + ro, p0);
    if (bxE) st4(S.psi[1][pn] + ro, p1);
}

// Samples of E(n+1/2) (full-grid ring copies and line samples).
__device__ __forceinline__ void te3_sample_e(const mtb_yee2d_struct &S, int i, int jb,
                                             uint32_t ro, const Ctx2D &C,
                                             const mtb_line_sample *L, int nl,
                                             const float (&ex)[4], const float (&ey)[4]) {
    float *ring = C.ring;
    if (S.ring_full[1] >= 0) st4(ring + S.ring_full[1] + ro, ex);
    if (S.ring_full[2] >= 0) st4(ring + S.ring_full[2] + ro, ey);
    if (nl) {
        sample_row(L, nl, MTB_C2_X, i, jb, true, ex, ring);
        sample_row(L, nl, MTB_C2_Y, i, jb, true, ey, ring);
    }
}

// Pass 2: E(n+1/2) from D(n+1/2) and P(n+1/2), and the E samples (with chi2 / chi3 the
// first iterate rhs / eps, into the scratch boxes; the sweeps sample the last one).
__device__ __forceinline__ void te3_e_row(const mtb_yee2d_struct &S, const int i, const int c0,
                                          const Ctx2D &C, const mtb_line_sample *L,
                                          const int nl) {
    const int lane = threadIdx.x;
    const int nx = S.nx, ny = S.ny, P = S.pitch;
    const int jb = c0 + 4 * lane;
    if (jb >= P) return;
    const int pn = C.par ^ 1;
    const uint32_t ro = (uint32_t)i * P + jb, pl = (uint32_t)nx * P;
    const float *Dx = S.f_x[pn], *Dy = S.f_y[pn];
    const int slot = (C.pst + 1) % 3;
    const float *Px = S.pol_p[slot], *Py = S.pol_py[slot];
    const int npx = S.n_poles, npy = S.n_poles_y;
    const bool tens = S.tinv[0] != nullptr, hasr = jb + 4 < P;
    float ex[4], ey[4];
    zero4(ex); zero4(ey);
    float rx[4], ry[4];
    zero4(rx);
    if (i <= nx - 2) te3_rhs4(Dx, Px, npx, pl, ro, rx);
    te3_rhs4(Dy, Py, npy, pl, ro, ry);
    if (tens) {
        float t0[4], t1[4], t2[4], t3[4];
        ld4(S.tinv[0] + ro, t0); ld4(S.tinv[1] + ro, t1);
        ld4(S.tinv[2] + ro, t2); ld4(S.tinv[3] + ro, t3);
        if (i <= nx - 2) {
            float ry1[4], ax[4];
            float l0 = jb >= 1 ? te3_rhs1(Dy, Py, npy, pl, ro - 1) : 0.f, l1 = 0.f;
            zero4(ry1);
            if (i + 1 < nx) {
                te3_rhs4(Dy, Py, npy, pl, ro + P, ry1);
                if (jb >= 1) l1 = te3_rhs1(Dy, Py, npy, pl, ro + P - 1);
            }
            te3_avg_ex(ry, l0, ry1, l1, jb, ny, ax);
#pragma unroll
            for (int q = 0; q < 4; ++q) ex[q] = t0[q] * rx[q] + t1[q] * ax[q];
        }
        float rxp[4], ay[4], pr = 0.f, cr = 0.f;
        zero4(rxp);
        if (i >= 1 && i - 1 <= nx - 2) {
            te3_rhs4(Dx, Px, npx, pl, ro - P, rxp);
            if (hasr) pr = te3_rhs1(Dx, Px, npx, pl, ro - P + 4);
        }
        if (i <= nx - 2 && hasr) cr = te3_rhs1(Dx, Px, npx, pl, ro + 4);
        te3_avg_ey(rxp, pr, rx, cr, ay);
#pragma unroll
        for (int q = 0; q < 4; ++q) ey[q] = t2[q] * ry[q] + t3[q] * ay[q];
    } else if (S.nlx[0]) {
        float epx[4], epy[4];                           // chi: rhs / eps, divided
        ld4(S.nlx[2] + ro, epx);
        ld4(S.nly[2] + ro, epy);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            ex[q] = __fdiv_rn(rx[q], epx[q]);
            ey[q] = __fdiv_rn(ry[q], epy[q]);
        }
    } else {
        float ix[4], iy[4];
        ld4(S.inv_eps_a + ro, ix);
        ld4(S.inv_eps_b + ro, iy);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            ex[q] = rx[q] * ix[q];
            ey[q] = ry[q] * iy[q];
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {                      // padding cells stay zero
        const int j = jb + q;
        if (!(i <= nx - 2 && j <= ny - 1)) ex[q] = 0.f;
        if (!(j <= ny - 2)) ey[q] = 0.f;
    }
    if (S.nlx[0]) {                                    // the sweeps go on from here
        st4(S.e_t[0] + ro, ex);
        st4(S.e_t[1] + ro, ey);
        return;
    }
    st4(S.e_x + ro, ex);
    st4(S.e_y + ro, ey);
    te3_sample_e(S, i, jb, ro, C, L, nl, ex, ey);
}

// One Jacobi sweep of the chi2 / chi3 fixed point (core/stepper_te.py:166-171): from the
// iterate in (ix_, iy_) to (ox, oy); E2 = E^2 + avg4(E_other)^2 of the input iterate.
// `last` samples the result.
__device__ __forceinline__ void te3_sweep_row(const mtb_yee2d_struct &S, const int i,
                                              const int c0, const Ctx2D &C,
                                              const mtb_line_sample *L, const int nl,
                                              const float *ix_, const float *iy_, float *ox,
                                              float *oy, bool last) {
    const int lane = threadIdx.x;
    const int nx = S.nx, ny = S.ny, P = S.pitch;
    const int jb = c0 + 4 * lane;
    if (jb >= P) return;
    const int pn = C.par ^ 1;
    const uint32_t ro = (uint32_t)i * P + jb, pl = (uint32_t)nx * P;
    const int slot = (C.pst + 1) % 3;
    const bool hasr = jb + 4 < P;
    float ex[4], ey[4], rx[4], ry[4], ax[4], ay[4];
    ld4(ix_ + ro, ex);
    ld4(iy_ + ro, ey);
    zero4(rx);
    if (i <= nx - 2) te3_rhs4(S.f_x[pn], S.pol_p[slot], S.n_poles, pl, ro, rx);
    te3_rhs4(S.f_y[pn], S.pol_py[slot], S.n_poles_y, pl, ro, ry);
    {
        float a1[4], l0 = jb >= 1 ? iy_[ro - 1] : 0.f, l1 = 0.f;
        zero4(a1);
        if (i + 1 < nx) {
            ld4(iy_ + ro + P, a1);
            if (jb >= 1) l1 = iy_[ro + P - 1];
        }
        te3_avg_ex(ey, l0, a1, l1, jb, ny, ax);
    }
    {
        float p[4], pr = 0.f, cr = 0.f;
        zero4(p);
        if (i >= 1 && i - 1 <= nx - 2) {
            ld4(ix_ + ro - P, p);
            if (hasr) pr = ix_[ro - P + 4];
        }
        if (i <= nx - 2 && hasr) cr = ix_[ro + 4];
        te3_avg_ey(p, pr, ex, cr, ay);
    }
    float x2[4], x3[4], xe[4], y2[4], y3[4], ye[4];
    ld4(S.nlx[0] + ro, x2); ld4(S.nlx[1] + ro, x3); ld4(S.nlx[2] + ro, xe);
    ld4(S.nly[0] + ro, y2); ld4(S.nly[1] + ro, y3); ld4(S.nly[2] + ro, ye);
    float nxv[4], nyv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        const float e2x = __fadd_rn(__fmul_rn(ex[q], ex[q]), __fmul_rn(ax[q], ax[q]));
        const float e2y = __fadd_rn(__fmul_rn(ey[q], ey[q]), __fmul_rn(ay[q], ay[q]));
        const float vx = __fdiv_rn(rx[q], __fadd_rn(__fadd_rn(xe[q], __fmul_rn(x2[q], ex[q])),
                                                    __fmul_rn(x3[q], e2x)));
        const float vy = __fdiv_rn(ry[q], __fadd_rn(__fadd_rn(ye[q], __fmul_rn(y2[q], ey[q])),
                                                    __fmul_rn(y3[q], e2y)));
        nxv[q] = (i <= nx - 2 && j <= ny - 1) ? vx : 0.f;  // padding cells stay zero
        nyv[q] = (j <= ny - 2) ? vy : 0.f;
    }
    st4(ox + ro, nxv);
    st4(oy + ro, nyv);
    if (last) te3_sample_e(S, i, jb, ro, C, L, nl, nxv, nyv);
}

// Pass 3: Hz(n+1) from the stored E(n+1/2) (core/stepper_te.py:103-117), its samples.
__device__ __forceinline__ void te3_h_row(const mtb_yee2d_struct &S, const int i, const int c0,
                                          const Ctx2D &C, const mtb_line_sample *L,
                                          const int nl) {
    const int lane = threadIdx.x;
    const int nx = S.nx, ny = S.ny, P = S.pitch;
    const int jb = c0 + 4 * lane;
    const bool act = jb < P;
    const float dt = S.dt, rdx = 1.0f / S.dx;
    const int par = C.par, pn = par ^ 1;
    const uint32_t ro = (uint32_t)i * P + (act ? jb : P - 4);
    const bool hzRow = i <= nx - 2;
    const bool bxH = hzRow && in_band(i, S.xband[0], S.xband[1]);
    const bool byH = act && hzRow && band4(jb, S.yband[0], S.yband[1]);
    float hc[4], ex[4], ey[4], eyn[4], p2[4], p3[4];
    zero4(hc); zero4(ex); zero4(ey); zero4(eyn); zero4(p2); zero4(p3);
    float exR = 0.f;
    if (act) {
        ld4(S.f_main[par] + ro, hc);
        ld4(S.e_x + ro, ex);
        ld4(S.e_y + ro, ey);
        if (i + 1 < nx) ld4(S.e_y + ro + P, eyn);
        if (lane == 31 && jb + 4 < P) exR = S.e_x[ro + 4];
        if (bxH) ld4(S.psi[2][par] + ro, p2);
        if (byH) ld4(S.psi[3][par] + ro, p3);
    }
    float exr = __shfl_down_sync(0xffffffffu, ex[0], 1);
    if (lane == 31) exr = exR;
    float hxb = 1.f, hxa = 0.f;
    if (bxH) { hxb = __ldg(S.hx_b + i); hxa = __ldg(S.hx_a + i); }
    const bool magz = S.mag_h1[0] != nullptr;
    float mz1[4] = {1.f, 1.f, 1.f, 1.f}, mz2[4] = {dt, dt, dt, dt};
    if (magz && act) {
        ld4(S.mag_h1[0] + ro, mz1);
        ld4(S.mag_h2[0] + ro, mz2);
    }
    float hzN[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        const bool v = act && hzRow && j <= ny - 2;
        const bool oh = byH && j <= ny - 2;
        const float hyb = oh ? __ldg(S.hy_b + j) : 1.f, hya = oh ? __ldg(S.hy_a + j) : 0.f;
        const float exn = (q < 3) ? ex[q + 1] : exr;
        const float dey = (eyn[q] - ey[q]) * rdx;
        const float dex = (exn - ex[q]) * rdx;
        const float q2 = hxb * p2[q] + hxa * dey;
        const float q3 = hyb * p3[q] + hya * dex;
        const float cz = (dey + q2) - (dex + q3);
        const float hn = magz ? mz1[q] * hc[q] - mz2[q] * cz : hc[q] - dt * cz;
        hzN[q] = v ? hn : hc[q];
        p2[q] = v ? q2 : p2[q];
        p3[q] = v ? q3 : p3[q];
    }
    if (act && hzRow && i >= S.src_h1.row_lo && i <= S.src_h1.row_hi)
        apply_cells(S.src_h1, i, C.amp_h, jb, hzN);
    if (!act) return;
    st4(S.f_main[pn] + ro, hzN);
    if (bxH) st4(S.psi[2][pn] + ro, p2);
    if (byH) st4(S.psi[3][pn] + ro, p3);
    float *ring = C.ring;
    if (S.ring_full[0] >= 0) st4(ring + S.ring_full[0] + ro, hzN);
    if (nl) sample_row(L, nl, MTB_C2_MAIN, i, jb, true, hzN, ring);
}

template <int PASS>
__global__ void __launch_bounds__(32 * TROWS, 2) k_te3(const mtb_yee2d_struct *__restrict__ SS,
                                                       const int4 *__restrict__ work,
                                                       int n_work, Ctx2D C) {
    __shared__ TileSmem T;
    int4 w;
    if (!tile_setup(SS, work, n_work, C.wr, T, w)) return;
    const mtb_yee2d_struct &S = T.s;
    const int ib = w.y + threadIdx.y * C.wr;
#pragma unroll 1
    for (int r = 0; r < C.wr; ++r) {
        const int i = ib + r;
        if (i >= S.nx) break;
        if (PASS == 0) te3_d_row(S, i, w.z, C);
        else if (PASS == 1) te3_e_row(S, i, w.z, C, T.lines, T.nl);
        else if (PASS == 2) te3_h_row(S, i, w.z, C, T.lines, T.nl);
        // chi sweeps 1, 2, 3: scratch -> E -> scratch -> E
        else if (PASS == 3) te3_sweep_row(S, i, w.z, C, T.lines, T.nl, S.e_t[0], S.e_t[1],
                                          S.e_x, S.e_y, false);
        else if (PASS == 4) te3_sweep_row(S, i, w.z, C, T.lines, T.nl, S.e_x, S.e_y,
                                          S.e_t[0], S.e_t[1], false);
        else te3_sweep_row(S, i, w.z, C, T.lines, T.nl, S.e_t[0], S.e_t[1], S.e_x, S.e_y,
                           true);
    }
}

}  // namespace mtb
