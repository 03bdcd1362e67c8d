// Discrete adjoint of the 2D TM step for sm_100a: the exact transpose of the
// forward update (core/stepper_tm.py:234-254: B phase :85-128, D phase
// :130-166, update_pols :203-208, E = (D - sum P) / eps :221-231) with CPML
// (kappa = 1, PEC walls or TM PMC walls in y), electric conductivity (D' = d1 D + d2 curl), magnetic
// conductivity / permeability (H' = h1 H -/+ h2 curl) and dispersive ADE poles,
// and of the monitors' sampling (core/monitors.py:24-100). This is what torch
// autograd computes through the reference's run_tm (core/run.py:43-120); the
// source terms are additive constants and have no adjoint. TE takes the same
// conductivity, magnetic pairs and poles (Px on Ex, Py on Ey).
//
// Reverse of forward step t (state_t -> state_{t+1}), adjoint state A holding
// dJ/d state_{t+1} on entry and dJ/d state_t on exit, three kernels:
//   k_adj_tm_e   (Ez/Dz nodes) monitor samples of Ez_{t+1} into gEz;
//                E = D / eps:  gD = gDz + gEz / eps, g_eps -= gEz Ez_{t+1} / eps;
//                D += dt pad(curl): g_curl = dt gD on the interior; the two psi
//                recursions of the curl; writes gDz, g_psi2, g_psi3 and the
//                adjoints of dHy/dx (tmp0) and dHx/dy (tmp1).
//   k_adj_tm_h   (H nodes) monitor samples of H_{t+1/2} into gHx, gHy; the
//                transposed differences of tmp0 / tmp1; H += -/+ dt curl E
//                with its psi recursions; writes gHx, gHy, g_psi0, g_psi1 and
//                the adjoints of dEz/dx (tmp2) and dEz/dy (tmp3).
//   k_adj_tm_ez  (Ez nodes) gEz = transposed differences of tmp2 / tmp3 (plus, with
//                poles, what k_adj_tm_e left in gEz).
// k_adj_tm_ez of step q and k_adj_tm_e of step q-1 touch the same node only, so within
// a chunk they run as one launch (k_adj_tm_eze): two launches per reverse step.
// Poles, P(n+1) = c1 P(n) + c2 P(n-1) + c3 Ez(n) with Ez(n+1) = (Dz - sum P(n+1)) / eps:
// with gA = d J / d P(n+1), gB = d J / d P(n) on entry, gPn = gA - gEz(n+1) / eps, and
// on exit gA = c1 gPn + gB, gB = c2 gPn, gEz(n) gets sum_k c3 gPn.
// The monitor adjoint of a whole chunk comes first: DftState::expand fills
// ring slot q with dJ/d(sample of step t0+q) in the forward ring's layout, and
// the kernels add it back at the cells the forward kernels sampled.
#include <algorithm>

#include "mtb_common.cuh"

namespace mtb {

constexpr int AROWS = 8;          // rows per block (one warp per row)
constexpr int AMAXL = 16;         // line samples per structure (the forward plan's limit)

__device__ __forceinline__ void ldv(const float *p, float (&v)[4]) {
    const float4 x = *reinterpret_cast<const float4 *>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void stv(float *p, const float (&v)[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// The structure's line-sample descriptors, copied to shared memory once per block
// (every thread of the block reads them for each of its cells).
__device__ __forceinline__ const mtb_line_sample *stage_lines(const mtb_yee2d_struct &S,
                                                              mtb_line_sample *sl) {
    const int t = threadIdx.y * 32 + threadIdx.x;
    if (t < S.n_lines) sl[t] = S.lines[t];
    __syncthreads();
    return sl;
}

// Add the adjoint ring's values for the forward samples of component `comp`
// at row i, columns jb .. jb+3 (the transpose of the forward kernels'
// full-grid sample and line samples).
__device__ __forceinline__ void inject(const mtb_yee2d_struct &S, const mtb_line_sample *L,
                                       int comp, int i, int jb, uint32_t g,
                                       const float *__restrict__ radj, float (&v)[4]) {
    const int64_t rf = S.ring_full[comp];
    if (rf >= 0) {
        float r[4];
        ldv(radj + rf + g, r);
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] += r[q];
    }
    for (int l = 0; l < S.n_lines; ++l) {
        const mtb_line_sample ln = L[l];
        if (ln.comp != comp) continue;
        if (ln.kind == 0) {
            if (ln.index != i) continue;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j = jb + q;
                if (j >= ln.lo && j < ln.hi) v[q] += radj[ln.ring_off + (j - ln.lo)];
            }
        } else {
            if (i < ln.lo || i >= ln.hi) continue;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (jb + q == ln.index) v[q] += radj[ln.ring_off + (i - ln.lo)];
        }
    }
}

__device__ __forceinline__ void adj_tm_e_cell(const mtb_yee2d_struct &S, const mtb_adj2d_buffers &B,
                                              const mtb_line_sample *L,
                                              const float *__restrict__ radj,
                                              const float *__restrict__ rec, const int i,
                                              const int jb, const int cpar) {
    const int nx = S.nx, ny = S.ny, P = S.pitch;
    if (i >= nx || jb >= P) return;
    const uint32_t g = (uint32_t)i * P + jb;
    const float dt = S.dt;
    float gez[4], gdz[4], gp2[4], gp3[4], ez[4], ie[4], ge[4];
    ldv(B.g[0] + g, gez);
    ldv(B.g[3] + g, gdz);
    ldv(B.g_psi[2] + g, gp2);
    ldv(B.g_psi[3] + g, gp3);
    ldv(rec + g, ez);
    ldv(S.inv_eps_a + g, ie);
    ldv(B.g_eps[0] + g, ge);
    inject(S, L, MTB_C2_MAIN, i, jb, g, radj, gez);
    // an even x mirror (cut_x 1, zero H ghost beyond the cut) makes the cut row live
    const bool rowin = (i >= 1 || S.cut_x) && i <= nx - 2;
    float bex = 1.f, aex = 0.f;
    if (rowin) { bex = S.ex_b[i]; aex = S.ex_a[i]; }
    // electric conductivity: D' = d1 D + d2 pad(curl)
    float d1[4] = {1.f, 1.f, 1.f, 1.f}, d2[4] = {dt, dt, dt, dt};
    if (S.cond_d1[0]) { ldv(S.cond_d1[0] + g, d1); ldv(S.cond_d2[0] + g, d2); }
    // poles: the gradient of P(n+1) and its transpose through the ADE recursion
    float gpe[4] = {0.f, 0.f, 0.f, 0.f};            // sum_k c3 gPn -> gEz(n)
    if (S.n_poles > 0) {
        const uint32_t pl = (uint32_t)nx * P;
        for (int k = 0; k < S.n_poles; ++k) {
            const uint32_t o = k * pl + g;
            float ga[4], gb[4], c1[4], c2[4], c3[4];
            ldv(B.g_pol[0] + o, ga);
            ldv(B.g_pol[1] + o, gb);
            ldv(S.pol_c[0] + o, c1);
            ldv(S.pol_c[1] + o, c2);
            ldv(S.pol_c[2] + o, c3);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float gpn = ga[q] - gez[q] * ie[q];
                ga[q] = c1[q] * gpn + gb[q];
                gb[q] = c2[q] * gpn;
                gpe[q] += c3[q] * gpn;
            }
            stv(B.g_pol[0] + o, ga);
            stv(B.g_pol[1] + o, gb);
        }
    }
    float t1[4], t2[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        const bool inside = j < ny;
        // the curl of the D update: interior columns, every column under PMC walls in y
        // (zero H beyond both walls, core/stepper_tm.py:143-145), or from the cut column
        // up under an even y mirror (zero H ghost beyond the cut, :146-148)
        const bool interior = rowin && (S.y_pmc ? j < ny : ((j >= 1 || S.cut_y) && j <= ny - 2));
        const float gd = gdz[q] + gez[q] * ie[q];
        ge[q] -= gez[q] * ez[q] * ie[q];
        const float gc = interior ? d2[q] * gd : 0.f;
        const float g2 = gp2[q] + gc, g3 = gp3[q] - gc;
        const float bey = interior ? S.ey_b[j] : 1.f, aey = interior ? S.ey_a[j] : 0.f;
        t1[q] = interior ? gc + aex * g2 : 0.f;
        t2[q] = interior ? -gc + aey * g3 : 0.f;
        gp2[q] = interior ? bex * g2 : gp2[q];
        gp3[q] = interior ? bey * g3 : gp3[q];
        gdz[q] = inside ? d1[q] * gd : 0.f;
        gpe[q] = inside ? gpe[q] : 0.f;
    }
    // live on-plane H lines (core/stepper_tm.py:100-115, :139-152): the cut row / column
    // of Dz differences against Hx0 / Hy0, so d J / d line(n+1/2) = (the next step's,
    // buffer cpar ^ 1) - (the difference adjoint) / dx, into buffer cpar
    if (S.cut_y == 2 && jb == 0)
        B.g_cut[0][cpar][i] = B.g_cut[0][cpar ^ 1][i] - t2[0] / S.dx;
    if (S.cut_x == 2 && i == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (jb + q < ny) B.g_cut[1][cpar][jb + q] = B.g_cut[1][cpar ^ 1][jb + q] - t1[q] / S.dx;
    if (S.n_poles > 0) stv(B.g[0] + g, gpe);     // gEz(n) from the poles; k_adj_tm_ez adds
    stv(B.g[3] + g, gdz);
    stv(B.g_psi[2] + g, gp2);
    stv(B.g_psi[3] + g, gp3);
    stv(B.tmp[0] + g, t1);
    stv(B.tmp[1] + g, t2);
    stv(B.g_eps[0] + g, ge);
}

__global__ void __launch_bounds__(32 * AROWS) k_adj_tm_e(const __grid_constant__ mtb_yee2d_struct S,
                                                         const __grid_constant__ mtb_adj2d_buffers B,
                                                         const float *__restrict__ radj,
                                                         const float *__restrict__ rec, int cpar) {
    __shared__ mtb_line_sample sl[AMAXL];
    const mtb_line_sample *L = stage_lines(S, sl);
    adj_tm_e_cell(S, B, L, radj, rec, blockIdx.y * AROWS + threadIdx.y,
                  (blockIdx.x * 32 + threadIdx.x) * 4, cpar);
}

__device__ __forceinline__ void adj_tm_h_cell(const mtb_yee2d_struct &S, const mtb_adj2d_buffers &B,
                                              const mtb_line_sample *L,
                                              const float *__restrict__ radj, const int i,
                                              const int jb) {
    const int nx = S.nx, ny = S.ny, P = S.pitch;
    if (i >= nx || jb >= P) return;
    const uint32_t g = (uint32_t)i * P + jb;
    const float dt = S.dt, rdx = 1.0f / S.dx;
    float ghx[4], ghy[4], gp0[4], gp1[4], t1[4], t1n[4], t2[4];
    ldv(B.g[1] + g, ghx);
    ldv(B.g[2] + g, ghy);
    ldv(B.g_psi[0] + g, gp0);
    ldv(B.g_psi[1] + g, gp1);
    ldv(B.tmp[0] + g, t1);
    ldv(B.tmp[1] + g, t2);
    if (i + 1 < nx) ldv(B.tmp[0] + g + P, t1n);
    else t1n[0] = t1n[1] = t1n[2] = t1n[3] = 0.f;
    const float t2r = (jb + 4 < P) ? B.tmp[1][g + 4] : 0.f;
    inject(S, L, MTB_C2_X, i, jb, g, radj, ghx);
    inject(S, L, MTB_C2_Y, i, jb, g, radj, ghy);
    const bool vrow = i <= nx - 2;
    float bhx = 1.f, ahx = 0.f;
    if (vrow) { bhx = S.hx_b[i]; ahx = S.hx_a[i]; }
    // magnetic conductivity / permeability: Hx' = h1 Hx - h2 curl, Hy' = h1 Hy + h2 curl
    float h1x[4] = {1.f, 1.f, 1.f, 1.f}, h2x[4] = {dt, dt, dt, dt};
    float h1y[4] = {1.f, 1.f, 1.f, 1.f}, h2y[4] = {dt, dt, dt, dt};
    if (S.mag_h1[0]) { ldv(S.mag_h1[0] + g, h1x); ldv(S.mag_h2[0] + g, h2x); }
    if (S.mag_h1[1]) { ldv(S.mag_h1[1] + g, h1y); ldv(S.mag_h2[1] + g, h2y); }
    float gxa[4], gya[4];                          // d J / d H(n+1/2)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float t2n = (q < 3) ? t2[q + 1] : t2r;
        gya[q] = ghy[q] + (t1[q] - t1n[q]) * rdx;
        gxa[q] = ghx[q] + (t2[q] - t2n) * rdx;
    }
    // magnetic poles (core/stepper_tm.py:209-219): B' = B -/+ dt curl, M(n+1) = mc1 M(n)
    // + mc2 M(n-1) + mc3 H(n-1/2), H(n+1/2) = B' - sum M(n+1). gN = gM(n)' - gH' per pole;
    // gM(n) = mc1 gN + gM(n-1)', gM(n-1) = mc2 gN, H(n-1/2) gets sum mc3 gN (its only use),
    // and the curl sees gB' + gH'
    const bool mp = S.n_mpoles > 0;
    float hxo[4] = {0.f, 0.f, 0.f, 0.f}, hyo[4] = {0.f, 0.f, 0.f, 0.f};
    if (mp) {
        float gbx[4], gby[4];
        ldv(B.g_b[0] + g, gbx);
        ldv(B.g_b[1] + g, gby);
        const uint32_t pl = (uint32_t)nx * P;
        for (int c = 0; c < 2; ++c) {
            const float(&gh)[4] = c ? gya : gxa;
            float(&acc)[4] = c ? hyo : hxo;
            for (int k = 0; k < S.n_mpoles; ++k) {
                const uint32_t o = k * pl + g;
                float ga[4], gb[4], m1[4], m2[4], m3[4];
                ldv(B.g_mpol[c][0] + o, ga); ldv(B.g_mpol[c][1] + o, gb);
                ldv(S.mpc[c][0] + o, m1); ldv(S.mpc[c][1] + o, m2); ldv(S.mpc[c][2] + o, m3);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float gn = ga[q] - gh[q];
                    ga[q] = m1[q] * gn + gb[q];
                    gb[q] = m2[q] * gn;
                    acc[q] += m3[q] * gn;
                }
                stv(B.g_mpol[c][0] + o, ga); stv(B.g_mpol[c][1] + o, gb);
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) { gxa[q] += gbx[q]; gya[q] += gby[q]; }
    }
    float t3[4], t4[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        const float gyp = gya[q], gxp = gxa[q];
        const bool vy = vrow && j < ny, vx = j <= ny - 2;
        // Hy = h1 Hy + h2 (dEz/dx + psi_Ezx'), psi_Ezx' = b_hx psi + a_hx dEz/dx
        const float cy = h2y[q] * gyp;
        const float g1 = gp1[q] + cy;
        t3[q] = vy ? cy + ahx * g1 : 0.f;
        gp1[q] = vy ? bhx * g1 : gp1[q];
        ghy[q] = vy ? (mp ? hyo[q] : h1y[q] * gyp) : 0.f;
        gya[q] = vy ? gyp : 0.f;                       // d J / d B(n-1/2) with poles
        // Hx = h1 Hx - h2 (dEz/dy + psi_Ezy'), psi_Ezy' = b_hy psi + a_hy dEz/dy
        const float bhy = vx ? S.hy_b[j] : 1.f, ahy = vx ? S.hy_a[j] : 0.f;
        const float cx = -h2x[q] * gxp;
        const float g0 = gp0[q] + cx;
        t4[q] = vx ? cx + ahy * g0 : 0.f;
        gp0[q] = vx ? bhy * g0 : gp0[q];
        ghx[q] = vx ? (mp ? hxo[q] : h1x[q] * gxp) : 0.f;
        gxa[q] = vx ? gxp : 0.f;
    }
    if (mp) { stv(B.g_b[0] + g, gxa); stv(B.g_b[1] + g, gya); }
    stv(B.g[1] + g, ghx);
    stv(B.g[2] + g, ghy);
    stv(B.g_psi[0] + g, gp0);
    stv(B.g_psi[1] + g, gp1);
    stv(B.tmp[2] + g, t3);
    stv(B.tmp[3] + g, t4);
}

__global__ void __launch_bounds__(32 * AROWS) k_adj_tm_h(const __grid_constant__ mtb_yee2d_struct S,
                                                         const __grid_constant__ mtb_adj2d_buffers B,
                                                         const float *__restrict__ radj) {
    __shared__ mtb_line_sample sl[AMAXL];
    const mtb_line_sample *L = stage_lines(S, sl);
    adj_tm_h_cell(S, B, L, radj, blockIdx.y * AROWS + threadIdx.y,
                  (blockIdx.x * 32 + threadIdx.x) * 4);
}

__device__ __forceinline__ void adj_tm_ez_cell(const mtb_yee2d_struct &S,
                                               const mtb_adj2d_buffers &B, const int i,
                                               const int jb, const int cpar) {
    const int nx = S.nx, ny = S.ny, P = S.pitch;
    if (i >= nx || jb >= P) return;
    const uint32_t g = (uint32_t)i * P + jb;
    const float rdx = 1.0f / S.dx;
    float t3[4], t3p[4], t4[4];
    ldv(B.tmp[2] + g, t3);
    if (i >= 1) ldv(B.tmp[2] + g - P, t3p);
    else t3p[0] = t3p[1] = t3p[2] = t3p[3] = 0.f;
    ldv(B.tmp[3] + g, t4);
    const float t4l = (jb >= 1) ? B.tmp[3][g - 1] : 0.f;
    float gez[4] = {0.f, 0.f, 0.f, 0.f};
    if (S.n_poles > 0) ldv(B.g[0] + g, gez);      // the poles' share, from k_adj_tm_e
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float t4m = (q == 0) ? t4l : t4[q - 1];
        gez[q] = (jb + q < ny) ? gez[q] + ((t3p[q] - t3[q]) * rdx + (t4m - t4[q]) * rdx) : 0.f;
    }
    // the on-plane H line updates of this step read Ez(n) (core/stepper_tm.py:100-115):
    //   Hx0' = Hx0 - dt (Ez(i, 0) - ph_y Ez(partner)) / dx, partner (i, 0), (nx-1-i, 0) or (0, i)
    //   Hy0' = Hy0 + dt (Ez(0, j) - ph_x Ez(partner)) / dx, partner (0, j) or (j, 0)
    if ((S.cut_y == 2 && (i == 0 || jb == 0)) || (S.cut_x == 2 && (i == 0 || jb == 0))) {
        const float k = S.dt * rdx;
        const float *gx = B.g_cut[0][cpar], *gy = B.g_cut[1][cpar];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = jb + q;
            if (j >= ny) continue;
            float a = 0.f;
            if (S.cut_y == 2) {
                const float ph = S.cut_ph_y;
                if (j == 0) {
                    a -= k * gx[i];
                    if (S.cut_map_y == 0) a += k * ph * gx[i];
                    else if (S.cut_map_y == 1) a += k * ph * gx[nx - 1 - i];
                }
                if (S.cut_map_y == 2 && i == 0 && j < nx) a += k * ph * gx[j];
            }
            if (S.cut_x == 2) {
                const float ph = S.cut_ph_x;
                if (i == 0) {
                    a += k * gy[j];
                    if (S.cut_map_x == 0) a -= k * ph * gy[j];
                }
                if (S.cut_map_x == 2 && j == 0 && i < ny) a -= k * ph * gy[i];
            }
            gez[q] += a;
        }
    }
    stv(B.g[0] + g, gez);
}

__global__ void __launch_bounds__(32 * AROWS) k_adj_tm_ez(const __grid_constant__ mtb_yee2d_struct S,
                                                          const __grid_constant__ mtb_adj2d_buffers B,
                                                          int cpar) {
    adj_tm_ez_cell(S, B, blockIdx.y * AROWS + threadIdx.y,
                  (blockIdx.x * 32 + threadIdx.x) * 4, cpar);
}

// ------------------------------------------------------------------ TE
// Reverse of TE step t (core/stepper_te.py:178-190: D from Hz(n), E = D / eps,
// Hz from E(n+1/2)), state_{t+1} = (Hz_{t+1}, E/D_{t+1/2}):
//   k_adj_te_h   (Hz nodes) samples of Hz_{t+1} into gHz; Hz -= dt ((dEy/dx + psi2')
//                - (dEx/dy + psi3')): g_psi2, g_psi3 and the adjoints of the two E
//                differences (tmp0 dEy/dx, tmp1 dEx/dy); gHz passes through.
//   k_adj_te_e   (E nodes) samples of Ex, Ey into gEx, gEy; transposed differences of
//                tmp0 / tmp1; E = D / eps: gD += gE / eps, g_eps -= gE E / eps (E of the
//                step from the record); D += dt (dHz/dy + psi0'), D -= dt (dHz/dx + psi1'):
//                g_psi0, g_psi1 and the adjoints of the two Hz differences (tmp2 at Dx
//                nodes, tmp3 at Dy nodes); gEx = gEy = 0 (E is recomputed every step).
//   k_adj_te_hz  (Hz nodes) gHz += transposed differences of tmp2 / tmp3.
// As for TM, k_adj_te_hz of step q and k_adj_te_h of step q-1 run as one launch
// (k_adj_te_hzh).
__device__ __forceinline__ void adj_te_h_cell(const mtb_yee2d_struct &S, const mtb_adj2d_buffers &B,
                                              const mtb_line_sample *L,
                                              const float *__restrict__ radj, const int i,
                                              const int jb) {
    const int nx = S.nx, ny = S.ny, P = S.pitch;
    if (i >= nx || jb >= P) return;
    const uint32_t g = (uint32_t)i * P + jb;
    const float dt = S.dt;
    float ghz[4], gp2[4], gp3[4];
    ldv(B.g[0] + g, ghz);
    ldv(B.g_psi[2] + g, gp2);
    ldv(B.g_psi[3] + g, gp3);
    inject(S, L, MTB_C2_MAIN, i, jb, g, radj, ghz);
    const bool vrow = i <= nx - 2;
    float hxb = 1.f, hxa = 0.f;
    if (vrow) { hxb = S.hx_b[i]; hxa = S.hx_a[i]; }
    // magnetic conductivity / permeability: Hz' = hz1 Hz - hz2 curl (core/stepper_te.py:112-114)
    float h1[4] = {1.f, 1.f, 1.f, 1.f}, h2[4] = {dt, dt, dt, dt};
    if (S.mag_h1[0]) { ldv(S.mag_h1[0] + g, h1); ldv(S.mag_h2[0] + g, h2); }
    float u0[4], u1[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        const bool v = vrow && j <= ny - 2;
        const float hyb = v ? S.hy_b[j] : 1.f, hya = v ? S.hy_a[j] : 0.f;
        const float c2 = -h2[q] * ghz[q], c3 = h2[q] * ghz[q];
        const float g2 = gp2[q] + c2, g3 = gp3[q] + c3;
        u0[q] = v ? c2 + hxa * g2 : 0.f;                  // dEy/dx
        u1[q] = v ? c3 + hya * g3 : 0.f;                  // dEx/dy
        gp2[q] = v ? hxb * g2 : gp2[q];
        gp3[q] = v ? hyb * g3 : gp3[q];
        ghz[q] = v ? h1[q] * ghz[q] : ghz[q];
    }
    stv(B.g[0] + g, ghz);
    stv(B.g_psi[2] + g, gp2);
    stv(B.g_psi[3] + g, gp3);
    stv(B.tmp[0] + g, u0);
    stv(B.tmp[1] + g, u1);
}

__global__ void __launch_bounds__(32 * AROWS) k_adj_te_h(const __grid_constant__ mtb_yee2d_struct S,
                                                         const __grid_constant__ mtb_adj2d_buffers B,
                                                         const float *__restrict__ radj) {
    __shared__ mtb_line_sample sl[AMAXL];
    const mtb_line_sample *L = stage_lines(S, sl);
    adj_te_h_cell(S, B, L, radj, blockIdx.y * AROWS + threadIdx.y,
                  (blockIdx.x * 32 + threadIdx.x) * 4);
}

__device__ __forceinline__ void adj_te_e_cell(const mtb_yee2d_struct &S, const mtb_adj2d_buffers &B,
                                              const mtb_line_sample *L,
                                              const float *__restrict__ radj,
                                              const float *__restrict__ rex,
                                              const float *__restrict__ rey, const int i,
                                              const int jb) {
    const int nx = S.nx, ny = S.ny, P = S.pitch;
    if (i >= nx || jb >= P) return;
    const uint32_t g = (uint32_t)i * P + jb;
    const float dt = S.dt, rdx = 1.0f / S.dx;
    float gex[4], gey[4], gdx[4], gdy[4], gp0[4], gp1[4], ex[4], ey[4], ix[4], iy[4];
    float u0[4], u0p[4], u1[4], gex_e[4], gey_e[4];
    ldv(B.g[1] + g, gex);
    ldv(B.g[2] + g, gey);
    ldv(B.g[3] + g, gdx);
    ldv(B.g[4] + g, gdy);
    ldv(B.g_psi[0] + g, gp0);
    ldv(B.g_psi[1] + g, gp1);
    ldv(rex + g, ex);
    ldv(rey + g, ey);
    ldv(S.inv_eps_a + g, ix);
    ldv(S.inv_eps_b + g, iy);
    ldv(B.g_eps[0] + g, gex_e);
    ldv(B.g_eps[1] + g, gey_e);
    ldv(B.tmp[0] + g, u0);
    ldv(B.tmp[1] + g, u1);
    if (i >= 1) ldv(B.tmp[0] + g - P, u0p);
    else u0p[0] = u0p[1] = u0p[2] = u0p[3] = 0.f;
    const float u1l = (jb >= 1) ? B.tmp[1][g - 1] : 0.f;
    inject(S, L, MTB_C2_X, i, jb, g, radj, gex);
    inject(S, L, MTB_C2_Y, i, jb, g, radj, gey);
    const bool xrow = i <= nx - 2, yrow = i >= 1 && i <= nx - 2;
    float exb = 1.f, exa = 0.f;
    if (yrow) { exb = S.ex_b[i]; exa = S.ex_a[i]; }
    // electric conductivity: Dx' = d1x Dx + d2x curl, Dy' = d1y Dy - d2y curl
    float dx1[4] = {1.f, 1.f, 1.f, 1.f}, dx2[4] = {dt, dt, dt, dt};
    float dy1[4] = {1.f, 1.f, 1.f, 1.f}, dy2[4] = {dt, dt, dt, dt};
    if (S.cond_d1[0]) {
        ldv(S.cond_d1[0] + g, dx1); ldv(S.cond_d2[0] + g, dx2);
        ldv(S.cond_d1[1] + g, dy1); ldv(S.cond_d2[1] + g, dy2);
    }
    float gX[4], gY[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        // Hz used dEx/dy = (Ex(j+1) - Ex(j)) and dEy/dx = (Ey(i+1) - Ey(i))
        const float u1m = (q == 0) ? u1l : u1[q - 1];
        gX[q] = xrow ? gex[q] + (u1m - u1[q]) * rdx : 0.f;   // Ex on rows <= nx-2 only
        gY[q] = gey[q] + (u0p[q] - u0[q]) * rdx;
    }
    // poles, E = (D - sum P(n+1)) / eps with P(n+1) = c1 P(n) + c2 P(n-1) + c3 E(n)
    // (core/stepper_te.py:136-175): gPn = gA - gE / eps, then gA = c1 gPn + gB,
    // gB = c2 gPn, and d J / d E(n) = sum_k c3 gPn (the next reverse step's gE)
    float pex[4] = {0.f, 0.f, 0.f, 0.f}, pey[4] = {0.f, 0.f, 0.f, 0.f};
    const uint32_t pl = (uint32_t)nx * P;
    for (int a = 0; a < 2; ++a) {
        const int np = a ? S.n_poles_y : S.n_poles;
        float *ga_ = a ? B.g_pol_y[0] : B.g_pol[0], *gb_ = a ? B.g_pol_y[1] : B.g_pol[1];
        const float *const *pc = a ? S.pol_cy : S.pol_c;
        const float(&gE)[4] = a ? gY : gX;
        const float(&ie)[4] = a ? iy : ix;
        float(&acc)[4] = a ? pey : pex;
        for (int k = 0; k < np; ++k) {
            const uint32_t o = k * pl + g;
            float ga[4], gb[4], c1[4], c2[4], c3[4];
            ldv(ga_ + o, ga); ldv(gb_ + o, gb);
            ldv(pc[0] + o, c1); ldv(pc[1] + o, c2); ldv(pc[2] + o, c3);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float gpn = ga[q] - gE[q] * ie[q];
                ga[q] = c1[q] * gpn + gb[q];
                gb[q] = c2[q] * gpn;
                acc[q] += c3[q] * gpn;
            }
            stv(ga_ + o, ga);
            stv(gb_ + o, gb);
        }
    }
    float t2[4], t3[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + q;
        // E = (D - sum P) / eps (Ex on rows <= nx-2 only)
        const float gdX = gdx[q] + (xrow ? gX[q] * ix[q] : 0.f);
        const float gdY = gdy[q] + gY[q] * iy[q];
        gex_e[q] -= xrow ? gX[q] * ex[q] * ix[q] : 0.f;
        gey_e[q] -= gY[q] * ey[q] * iy[q];
        // Dx' = d1x Dx + d2x (d + psi0'): the curl on i <= nx-2, 1 <= j <= ny-2; an even
        // y mirror adds the cut row j = 0 with curl 2 Hz / dx and no psi
        // (core/stepper_te.py:87-93), whose transpose is 2 c0 on the Hz difference slot
        const bool vx = xrow && j >= 1 && j <= ny - 2;
        const bool cy = xrow && j == 0 && S.cut_y == 1;
        const float eyb = vx ? S.ey_b[j] : 1.f, eya = vx ? S.ey_a[j] : 0.f;
        const float c0 = dx2[q] * gdX, g0 = gp0[q] + c0;
        t2[q] = vx ? c0 + eya * g0 : (cy ? 2.f * c0 : 0.f);
        gp0[q] = vx ? eyb * g0 : gp0[q];
        // Dy' = d1y Dy - d2y (d + psi1'): the curl on 1 <= i <= nx-2, j <= ny-2; an even
        // x mirror adds the cut row i = 0 the same way (:94-96)
        const bool vy = yrow && j <= ny - 2;
        const bool cx = i == 0 && S.cut_x == 1 && j <= ny - 2;
        const float c1 = -dy2[q] * gdY, g1 = gp1[q] + c1;
        t3[q] = vy ? c1 + exa * g1 : (cx ? 2.f * c1 : 0.f);
        gp1[q] = vy ? exb * g1 : gp1[q];
        gdx[q] = dx1[q] * gdX;
        gdy[q] = dy1[q] * gdY;
        // E(n) reaches J only through the poles' recursion
        gex[q] = xrow && j < ny ? pex[q] : 0.f;
        gey[q] = j <= ny - 2 ? pey[q] : 0.f;
    }
    stv(B.g[1] + g, gex);
    stv(B.g[2] + g, gey);
    stv(B.g[3] + g, gdx);
    stv(B.g[4] + g, gdy);
    stv(B.g_psi[0] + g, gp0);
    stv(B.g_psi[1] + g, gp1);
    stv(B.g_eps[0] + g, gex_e);
    stv(B.g_eps[1] + g, gey_e);
    stv(B.tmp[2] + g, t2);
    stv(B.tmp[3] + g, t3);
}

__global__ void __launch_bounds__(32 * AROWS) k_adj_te_e(const __grid_constant__ mtb_yee2d_struct S,
                                                         const __grid_constant__ mtb_adj2d_buffers B,
                                                         const float *__restrict__ radj,
                                                         const float *__restrict__ rex,
                                                         const float *__restrict__ rey) {
    __shared__ mtb_line_sample sl[AMAXL];
    const mtb_line_sample *L = stage_lines(S, sl);
    adj_te_e_cell(S, B, L, radj, rex, rey, blockIdx.y * AROWS + threadIdx.y,
                  (blockIdx.x * 32 + threadIdx.x) * 4);
}

__device__ __forceinline__ void adj_te_hz_cell(const mtb_yee2d_struct &S,
                                               const mtb_adj2d_buffers &B, const int i,
                                               const int jb) {
    const int nx = S.nx, ny = S.ny, P = S.pitch;
    if (i >= nx || jb >= P) return;
    const uint32_t g = (uint32_t)i * P + jb;
    const float rdx = 1.0f / S.dx;
    float ghz[4], t2[4], t3[4], t3n[4];
    ldv(B.g[0] + g, ghz);
    ldv(B.tmp[2] + g, t2);
    ldv(B.tmp[3] + g, t3);
    if (i + 1 < nx) ldv(B.tmp[3] + g + P, t3n);
    else t3n[0] = t3n[1] = t3n[2] = t3n[3] = 0.f;
    const float t2r = (jb + 4 < P) ? B.tmp[2][g + 4] : 0.f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float t2n = (q < 3) ? t2[q + 1] : t2r;
        const bool v = i <= nx - 2 && jb + q <= ny - 2;
        ghz[q] = v ? ghz[q] + (t2[q] - t2n) * rdx + (t3[q] - t3n[q]) * rdx : 0.f;
    }
    stv(B.g[0] + g, ghz);
}

__global__ void __launch_bounds__(32 * AROWS) k_adj_te_hz(const __grid_constant__ mtb_yee2d_struct S,
                                                          const __grid_constant__ mtb_adj2d_buffers B) {
    adj_te_hz_cell(S, B, blockIdx.y * AROWS + threadIdx.y,
                  (blockIdx.x * 32 + threadIdx.x) * 4);
}

// Two node-local kernels of consecutive reverse steps in one launch: the last kernel
// of step q (gEz / gHz from the neighbours' difference adjoints, written by the
// previous launch) and the first kernel of step q-1 on the same node, which reads only
// that node's adjoint state. Three launches per step become two.
__global__ void __launch_bounds__(32 * AROWS) k_adj_tm_eze(const __grid_constant__ mtb_yee2d_struct S,
                                                           const __grid_constant__ mtb_adj2d_buffers B,
                                                           const float *__restrict__ radj,
                                                           const float *__restrict__ rec, int cpar) {
    __shared__ mtb_line_sample sl[AMAXL];
    const mtb_line_sample *L = stage_lines(S, sl);
    const int i = blockIdx.y * AROWS + threadIdx.y, jb = (blockIdx.x * 32 + threadIdx.x) * 4;
    // cpar is the earlier step's buffer: this step's line gradient is in cpar ^ 1, which
    // no thread of this launch writes
    adj_tm_ez_cell(S, B, i, jb, cpar ^ 1);
    adj_tm_e_cell(S, B, L, radj, rec, i, jb, cpar);
}

__global__ void __launch_bounds__(32 * AROWS) k_adj_te_hzh(const __grid_constant__ mtb_yee2d_struct S,
                                                           const __grid_constant__ mtb_adj2d_buffers B,
                                                           const float *__restrict__ radj) {
    __shared__ mtb_line_sample sl[AMAXL];
    const mtb_line_sample *L = stage_lines(S, sl);
    const int i = blockIdx.y * AROWS + threadIdx.y, jb = (blockIdx.x * 32 + threadIdx.x) * 4;
    adj_te_hz_cell(S, B, i, jb);
    adj_te_h_cell(S, B, L, radj, i, jb);
}

}  // namespace mtb

using namespace mtb;

struct mtb_yee2d_adjoint {
    mtb_yee2d_struct s{};
    mtb_adj2d_buffers b{};
    DftState dft;
    int64_t last_launches = 0;
    // a whole chunk (ring_slots reverse steps with its sample adjoint) replayed
    // as a CUDA graph, valid for the forward record it was captured with
    cudaStream_t cap = nullptr;
    cudaGraphExec_t gexec = nullptr;
    const float *g_rec = nullptr;
    int64_t g_rec_slot = -1, g_rec_off[2] = {-1, -1}, gkern = 0;
};

// The device work of one chunk of k reverse steps on `st` (after the phases
// of its steps are uploaded).
static int adjoint_chunk(mtb_yee2d_adjoint *p, int k, const float *rec, int64_t rec_slot_elems,
                         const int64_t *rec_offset, cudaStream_t st) {
    int rc;
    if (p->dft.n_regions > 0) {
        if ((rc = p->dft.expand(0, k, st))) return rc;
        ++p->last_launches;
    } else {
        MTB_CUDA_TRY(cudaMemsetAsync(p->dft.ring_d.p, 0,
                                     sizeof(float) * (size_t)p->dft.slot_elems * k, st));
    }
    const mtb_yee2d_struct &S = p->s;
    const dim3 blk(32, AROWS);
    const dim3 grid((S.pitch / 4 + 31) / 32, (S.nx + AROWS - 1) / AROWS);
    // step q: first kernel (fused with the previous step's last, except at q = k-1),
    // middle kernel, and the last kernel alone only at q = 0
    auto radj_of = [&](int q) { return p->dft.ring_d.as<float>() + (size_t)q * p->dft.slot_elems; };
    auto rec_of = [&](int q) { return rec + (size_t)q * rec_slot_elems; };
    // live on-plane H lines: step q of the chunk writes line gradient buffer q & 1 and
    // reads the later step's from (q + 1) & 1; the previous chunk ended in buffer 0, so an
    // odd chunk starts with that copied to buffer 1 (device copies of nx / ny floats)
    if (S.pol == MTB_TM && (k & 1))
        for (int a = 0; a < 2; ++a)
            if ((a ? S.cut_x : S.cut_y) == 2)
                MTB_CUDA_TRY(cudaMemcpyAsync(p->b.g_cut[a][1], p->b.g_cut[a][0],
                                             sizeof(float) * (a ? S.ny : S.nx),
                                             cudaMemcpyDeviceToDevice, st));
    for (int q = k - 1; q >= 0; --q) {
        const float *radj = radj_of(q);
        const float *rq = rec_of(q);
        if (S.pol == MTB_TM) {
            if (q == k - 1) {
                k_adj_tm_e<<<grid, blk, 0, st>>>(S, p->b, radj, rq + rec_offset[0], q & 1);
                MTB_CHECK_LAUNCH();
            }
            k_adj_tm_h<<<grid, blk, 0, st>>>(S, p->b, radj);
            MTB_CHECK_LAUNCH();
            if (q > 0)
                k_adj_tm_eze<<<grid, blk, 0, st>>>(S, p->b, radj_of(q - 1),
                                                   rec_of(q - 1) + rec_offset[0], (q - 1) & 1);
            else
                k_adj_tm_ez<<<grid, blk, 0, st>>>(S, p->b, 0);
            MTB_CHECK_LAUNCH();
        } else {
            if (q == k - 1) {
                k_adj_te_h<<<grid, blk, 0, st>>>(S, p->b, radj);
                MTB_CHECK_LAUNCH();
            }
            k_adj_te_e<<<grid, blk, 0, st>>>(S, p->b, radj, rq + rec_offset[0], rq + rec_offset[1]);
            MTB_CHECK_LAUNCH();
            if (q > 0)
                k_adj_te_hzh<<<grid, blk, 0, st>>>(S, p->b, radj_of(q - 1));
            else
                k_adj_te_hz<<<grid, blk, 0, st>>>(S, p->b);
            MTB_CHECK_LAUNCH();
        }
        p->last_launches += (q == k - 1) ? 3 : 2;
    }
    return MTB_OK;
}

extern "C" {

int mtb_yee2d_adjoint_create(const mtb_yee2d_struct *s, const mtb_adj2d_buffers *bufs,
                             const mtb_dft_region *regions, int32_t n_regions,
                             const mtb_phase_group *groups, int32_t n_groups,
                             int64_t ring_slot_elems, int32_t ring_slots,
                             mtb_yee2d_adjoint **out) {
    if (!out || !s || !bufs) return fail(MTB_INVALID_ARG, "null argument");
    *out = nullptr;
    const mtb_yee2d_struct &S = *s;
    if (S.pol != MTB_TM && S.pol != MTB_TE) return fail(MTB_INVALID_ARG, "adjoint: bad pol");
    if (S.cut_y < 0 || S.cut_y > 2 || S.cut_x < 0 || S.cut_x > 2)
        return fail(MTB_INVALID_ARG, "adjoint: cut_y / cut_x must be 0, 1 or 2");
    for (int a = 0; a < 2; ++a)
        if ((a ? S.cut_x : S.cut_y) == 2 &&
            (S.pol != MTB_TM || !bufs->g_cut[a][0] || !bufs->g_cut[a][1]))
            return fail(MTB_INVALID_ARG, "adjoint: a live cut line needs TM and g_cut[%d][0..1]", a);
    if (S.cut_y && S.y_pmc) return fail(MTB_INVALID_ARG, "adjoint: cut_y with y_pmc");
    if (S.y_pmc && S.pol != MTB_TM) return fail(MTB_INVALID_ARG, "adjoint: y_pmc is TM only");
    if (S.chi2) return fail(MTB_UNSUPPORTED, "adjoint: chi2 / chi3 (a nonlinear step)");
    if (S.n_mpoles < 0 || S.n_mpoles > MTB_MAX_POLES ||
        (S.n_mpoles && (S.pol != MTB_TM || S.mag_h1[0] || S.mag_h1[1])))
        return fail(MTB_INVALID_ARG, "adjoint: n_mpoles %d (TM, without magnetic pairs)",
                    S.n_mpoles);
    if (S.n_mpoles)
        for (int c = 0; c < 2; ++c)
            if (!bufs->g_b[c] || !bufs->g_mpol[c][0] || !bufs->g_mpol[c][1] || !S.mpc[c][0] ||
                !S.mpc[c][1] || !S.mpc[c][2] || (reinterpret_cast<uintptr_t>(bufs->g_b[c]) & 15) ||
                (reinterpret_cast<uintptr_t>(bufs->g_mpol[c][0]) & 15) ||
                (reinterpret_cast<uintptr_t>(bufs->g_mpol[c][1]) & 15))
                return fail(MTB_INVALID_ARG, "adjoint: magnetic poles need g_b, g_mpol and mc1..3");
    if (S.te3) return fail(MTB_UNSUPPORTED, "adjoint: TE tensor eps / oriented poles");
    if (S.n_lines < 0 || S.n_lines > AMAXL || (S.n_lines > 0 && !S.lines))
        return fail(MTB_INVALID_ARG, "adjoint: %d line samples (at most %d)", S.n_lines, AMAXL);
    if ((S.cond_d1[0] && !S.cond_d2[0]) || (S.mag_h1[0] && !S.mag_h2[0]) ||
        (S.mag_h1[1] && !S.mag_h2[1]) ||
        (S.pol == MTB_TE && S.cond_d1[0] && (!S.cond_d1[1] || !S.cond_d2[1])))
        return fail(MTB_INVALID_ARG, "adjoint: damping pairs need both arrays");
    if (S.pol == MTB_TE && S.n_poles_y > 0 &&
        (!bufs->g_pol_y[0] || !bufs->g_pol_y[1] ||
         (reinterpret_cast<uintptr_t>(bufs->g_pol_y[0]) & 15) ||
         (reinterpret_cast<uintptr_t>(bufs->g_pol_y[1]) & 15) || !S.pol_cy[0] || !S.pol_cy[1] ||
         !S.pol_cy[2]))
        return fail(MTB_INVALID_ARG, "adjoint: Ey poles need g_pol_y[0..1] and c1..c3");
    if (S.n_poles > 0 && (!bufs->g_pol[0] || !bufs->g_pol[1] ||
                          (reinterpret_cast<uintptr_t>(bufs->g_pol[0]) & 15) ||
                          (reinterpret_cast<uintptr_t>(bufs->g_pol[1]) & 15) || !S.pol_c[0] ||
                          !S.pol_c[1] || !S.pol_c[2]))
        return fail(MTB_INVALID_ARG, "adjoint: poles need g_pol[0..1] and the c1..c3 arrays");
    if (S.nx < 3 || S.ny < 3 || S.pitch < S.ny || (S.pitch & 3))
        return fail(MTB_INVALID_ARG, "adjoint: bad grid %d x %d, pitch %d", S.nx, S.ny, S.pitch);
    if ((int64_t)S.nx * S.pitch >= (1LL << 31)) return fail(MTB_UNSUPPORTED, "grid too large");
    if (S.nx > 65535 * AROWS) return fail(MTB_UNSUPPORTED, "adjoint: nx too large");
    auto bad = [](const void *p) { return !p || (reinterpret_cast<uintptr_t>(p) & 15); };
    const bool te = S.pol == MTB_TE;
    for (int c = 0; c < 4; ++c)
        if (bad(bufs->g[c]) || bad(bufs->g_psi[c]) || bad(bufs->tmp[c]))
            return fail(MTB_INVALID_ARG, "adjoint: null or unaligned buffer");
    if ((te && bad(bufs->g[4])) || bad(bufs->g_eps[0]) || bad(S.inv_eps_a) ||
        (te && (bad(bufs->g_eps[1]) || bad(S.inv_eps_b))))
        return fail(MTB_INVALID_ARG, "adjoint: null or unaligned g / g_eps / inv_eps");
    if (!S.hx_b || !S.hx_a || !S.hy_b || !S.hy_a || !S.ex_b || !S.ex_a || !S.ey_b || !S.ey_a)
        return fail(MTB_INVALID_ARG, "adjoint: null CPML profile");
    if (S.n_lines < 0 || (S.n_lines > 0 && !S.lines))
        return fail(MTB_INVALID_ARG, "adjoint: bad line samples");
    for (int c = 0; c < 3; ++c) {
        const int64_t o = S.ring_full[c];
        if (o >= 0 && ((o & 3) || o + (int64_t)S.nx * S.pitch > ring_slot_elems))
            return fail(MTB_INVALID_ARG, "adjoint: full-grid ring offset %lld invalid",
                        (long long)o);
    }
    if (ring_slot_elems & 3) return fail(MTB_INVALID_ARG, "ring_slot_elems must be a multiple of 4");
    mtb_yee2d_adjoint *p = new mtb_yee2d_adjoint();
    p->s = S;
    p->b = *bufs;
    const int rc = p->dft.init(regions, n_regions, groups, n_groups, ring_slot_elems,
                               ring_slots > 0 ? ring_slots : 32);
    if (rc) { p->dft.release(); delete p; return rc; }
    // the adjoint ring must exist even without regions (line / full samples read it)
    if (n_regions == 0) {
        const int rc2 = p->dft.ring_d.ensure(sizeof(float) * (size_t)std::max<int64_t>(
                                                                ring_slot_elems, 4) * p->dft.slots);
        if (rc2) { p->dft.release(); delete p; return rc2; }
    }
    *out = p;
    return MTB_OK;
}

int mtb_yee2d_adjoint_run(mtb_yee2d_adjoint *p, int64_t t0, int32_t k, const float *rec,
                          int64_t rec_slot_elems, const int64_t *rec_offset_in, void *stream) {
    if (!p) return fail(MTB_INVALID_ARG, "adjoint plan is null");
    p->last_launches = 0;
    if (k <= 0) return MTB_OK;
    if (k > p->dft.slots) return fail(MTB_INVALID_ARG, "k %d > ring slots %d", k, p->dft.slots);
    if (!rec_offset_in) return fail(MTB_INVALID_ARG, "adjoint: null record offsets");
    const int64_t rec_offset[2] = {rec_offset_in[0],
                                   p->s.pol == MTB_TE ? rec_offset_in[1] : rec_offset_in[0]};
    if (!rec || (rec_offset[0] & 3) || (rec_offset[1] & 3) || rec_offset[0] < 0 ||
        rec_offset[1] < 0 || (rec_slot_elems & 3) || (reinterpret_cast<uintptr_t>(rec) & 15))
        return fail(MTB_INVALID_ARG, "adjoint: bad forward record");
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    if ((rc = p->dft.upload_phases(t0, k, st))) return rc;
    const bool whole = k == p->dft.slots;
    if (whole && !p->gexec) {                  // capture the whole-chunk graph once
        if (!p->cap) MTB_CUDA_TRY(cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking));
        const int64_t l0 = mtb_launch_count();
        MTB_CUDA_TRY(cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeThreadLocal));
        rc = adjoint_chunk(p, k, rec, rec_slot_elems, rec_offset, p->cap);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(p->cap, &g);
        const int64_t nk = mtb_launch_count() - l0;
        count_launch(-nk);                     // captured, not launched
        if (!rc && e != cudaSuccess)
            rc = fail(MTB_CUDA_ERROR, "adjoint graph capture: %s", cudaGetErrorString(e));
        if (!rc) {
            const cudaError_t ei = cudaGraphInstantiate(&p->gexec, g, 0);
            if (ei != cudaSuccess) {
                p->gexec = nullptr;
                rc = fail(MTB_CUDA_ERROR, "adjoint graph instantiate: %s", cudaGetErrorString(ei));
            }
        }
        if (g) cudaGraphDestroy(g);
        if (rc) return rc;
        p->gkern = nk;
        p->g_rec = rec;
        p->g_rec_slot = rec_slot_elems;
        p->g_rec_off[0] = rec_offset[0];
        p->g_rec_off[1] = rec_offset[1];
    }
    p->last_launches = 0;
    if (whole && p->gexec && p->g_rec == rec && p->g_rec_slot == rec_slot_elems &&
        p->g_rec_off[0] == rec_offset[0] && p->g_rec_off[1] == rec_offset[1]) {
        MTB_CUDA_TRY(cudaGraphLaunch(p->gexec, st));
        count_launch(p->gkern);
        p->last_launches = p->gkern;
        return MTB_OK;
    }
    return adjoint_chunk(p, k, rec, rec_slot_elems, rec_offset, st);
}

int64_t mtb_yee2d_adjoint_last_launches(const mtb_yee2d_adjoint *p) {
    return p ? p->last_launches : -1;
}

void mtb_yee2d_adjoint_destroy(mtb_yee2d_adjoint *p) {
    if (!p) return;
    if (p->gexec) cudaGraphExecDestroy(p->gexec);
    if (p->cap) cudaStreamDestroy(p->cap);
    p->dft.release();
    delete p;
}

}  // extern "C"
