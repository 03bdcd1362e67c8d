// Discrete adjoint of the 3D CPML step for sm_100a (with conductive damping:
// H' = d1 H - d2 curl, E' = d1 E + d2 curl / eps, dispersive poles, whose
// recurrence is linear with eps-free coefficients, and PMC walls): the exact transpose of
// the split H / E update (core/stepper_3d.py:363-437, the same arithmetic as
// k_yee3d_h / k_yee3d_e) and of the plane sampling (core/monitors_3d.py:70-189)
// -- the reverse sweep of the reference's run_3d_adjoint
// (core/adjoint3d.py:56-115). Sources are additive constants; their only
// derivative is through eps (E += s / eps_c), which the E-increment form below
// carries.
//
// Reverse of forward step t, adjoint state A = d J / d state_{t+1} on entry:
//   k_adj3_inject  monitor plane samples of state_{t+1} -> gE, gH (scatter)
//   k_adj3_e       E' = E + (dt curl + s) / eps_c:
//                    d J / d eps_c = -gE' (E' - E) / eps_c       -> tmp6..8
//                    g_curl = dt gE' / eps_c on the curl interior
//                    E-side psi transposes -> g_psi6..11, adjoints of the six
//                    H differences -> tmp0..5; gE passes through (identity)
//   k_adj3_h       gH += transposed differences of tmp0..5; H' = H - dt curl E:
//                    H-side psi transposes -> g_psi0..5, adjoints of the six E
//                    differences -> tmp9..14
//   k_adj3_fin     gE += transposed differences of tmp9..14;
//                  g_eps += the two cells of each Yee average (tmp6..8)
// tmp index: 0 Ex:dy(Hz) 1 Ex:dz(Hy) 2 Ey:dz(Hx) 3 Ey:dx(Hz) 4 Ez:dx(Hy)
// 5 Ez:dy(Hx) 6 eps_x 7 eps_y 8 eps_z 9 Hx:dy(Ez) 10 Hx:dz(Ey) 11 Hy:dz(Ex)
// 12 Hy:dx(Ez) 13 Hz:dx(Ey) 14 Hz:dy(Ex); a tmp array is zero outside the
// cells where its term exists.
#include <algorithm>
#include <vector>

#include "mtb_common.cuh"

namespace mtb {

constexpr int A3Y = 8;            // y rows per block (warp = 128 z of one row)

struct Adj3 {
    mtb_adj3d_buffers b;
    const float *eps;
    const float *pb[3][2];
    const float *pa[3][2];
    const float *dmp[6][2];       // conductive damping (d1, d2) per component, or null
    const float *c3[3];           // pole drives per E component (np box planes each)
    float c1[MTB_MAX_POLES], c2[MTB_MAX_POLES];
    int np;                       // dispersive poles (0: none)
    int pmc;                      // PMC walls: bit 0 x, 1 y, 2 z
    int nx, ny, nz, zp;
    float dt, rdx;
};

__device__ __forceinline__ void l4(const float *p, float (&v)[4]) {
    const float4 x = *reinterpret_cast<const float4 *>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void s4(float *p, const float (&v)[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void zz(float (&v)[4]) { v[0] = v[1] = v[2] = v[3] = 0.f; }
__device__ __forceinline__ float prof(const float *p, bool on, float dflt, int k) {
    return on ? __ldg(p + k) : dflt;
}

// gF[cell] += adjoint ring value, for every plane sample of the step.
__global__ void k_adj3_inject(const mtb_yee3d_struct *__restrict__ SS,
                              const int64_t *__restrict__ pstart, int n_planes,
                              const float *__restrict__ radj, mtb_adj3d_buffers B) {
    const mtb_yee3d_struct &S = *SS;
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= pstart[n_planes]) return;
    int lo = 0, hi = n_planes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pstart[mid] <= e) lo = mid; else hi = mid - 1;
    }
    const int *pl = S.planes + 8 * lo;
    const int comp = pl[0], axis = pl[1], index = pl[2];
    const int w1 = pl[6] - pl[5];
    const int64_t p = e - pstart[lo];
    const int a = pl[3] + (int)(p / w1), b = pl[5] + (int)(p % w1);
    int i, j, k;
    if (axis == 0) { i = index; j = a; k = b; }
    else if (axis == 1) { i = a; j = index; k = b; }
    else { i = a; j = b; k = index; }
    atomicAdd(B.g[comp] + ((int64_t)i * S.ny + j) * S.zpitch + k,
              radj[S.plane_ring_off[lo] + p]);
}

__global__ void __launch_bounds__(32 * A3Y) k_adj3_e(const __grid_constant__ Adj3 P,
                                                    const float *__restrict__ en_,
                                                    const float *__restrict__ eo_,
                                                    int64_t rec_comp) {
    const int nx = P.nx, ny = P.ny, nz = P.nz, ZP = P.zp;
    const int lane = threadIdx.x;
    const int j = blockIdx.y * A3Y + threadIdx.y;
    const int i = blockIdx.z;
    const int kb = blockIdx.x * 128 + 4 * lane;
    const bool act = j < ny && kb < ZP;
    const uint32_t NYZ = (uint32_t)ny * ZP;
    const uint32_t g = (uint32_t)i * NYZ + (uint32_t)(j * ZP + kb);
    const mtb_adj3d_buffers &B = P.b;
    const float dt = P.dt;
    float ep[4], epi[4], epj[4], epk = 1.f;
    ep[0] = ep[1] = ep[2] = ep[3] = 1.f;
    epi[0] = epi[1] = epi[2] = epi[3] = 1.f;
    epj[0] = epj[1] = epj[2] = epj[3] = 1.f;
    if (act) {
        l4(P.eps + g, ep);
        if (i + 1 < nx) l4(P.eps + g + NYZ, epi);
        if (j + 1 < ny) l4(P.eps + g + ZP, epj);
        if (lane == 31 && kb + 4 < ZP) epk = P.eps[g + 4];
    }
    {
        const float t = __shfl_down_sync(0xffffffffu, ep[0], 1);
        if (lane != 31) epk = t;
    }
    if (!act) return;
    const bool iin = i >= 1 && i <= nx - 2, jin = j >= 1 && j <= ny - 2;
    const bool xok = i <= nx - 2, vyH = j <= ny - 2;
    float ge[3][4], en[3][4], eo[3][4], gp[6][4];
    for (int c = 0; c < 3; ++c) {
        l4(B.g[c] + g, ge[c]);
        l4(en_ + c * rec_comp + g, en[c]);
        l4(eo_ + c * rec_comp + g, eo[c]);
    }
    for (int c = 0; c < 6; ++c) l4(B.g_psi[6 + c] + g, gp[c]);
    // conductive damping: E' = d1 E + (d2 curl + s) / eps_c (core/stepper_3d.py:405-437)
    const bool damp = P.dmp[0][0] != nullptr;
    float d1[3][4], d2[3][4];
    for (int c = 0; c < 3; ++c)
        for (int q = 0; q < 4; ++q) { d1[c][q] = 1.f; d2[c][q] = dt; }
    if (damp)
        for (int c = 0; c < 3; ++c) { l4(P.dmp[c][0] + g, d1[c]); l4(P.dmp[c][1] + g, d2[c]); }
    // dispersive poles (core/stepper_3d.py:295-300, :311-322): P(n+1) = c1 P(n) +
    // c2 P(n-1) + c3 E(n), E' = (d1 (E eps_c + sum P(n)) + d2 curl + s - sum P(n+1)) / eps_c.
    // P(n+1) is the next state's P(n), so gN = d J / d P(n+1) = gPc' - gE' / eps_c, and
    //   d J / d E(n) gains sum c3 gN,  gPc = d1 gE' / eps_c + c1 gN + gPp',  gPp = c2 gN.
    float pe[3][4];
    for (int c = 0; c < 3; ++c) zz(pe[c]);
    if (P.np > 0) {
        const size_t plane = (size_t)nx * NYZ;
        for (int c = 0; c < 3; ++c) {
            float ec[4];
            bool pv[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int k = kb + q;
                const float o = c == 0 ? epi[q] : c == 1 ? epj[q] : (q < 3 ? ep[q + 1] : epk);
                ec[q] = 0.5f * (ep[q] + o);
                pv[q] = c == 0 ? (xok && k < nz) : c == 1 ? (vyH && k < nz) : (k <= nz - 2);
            }
            for (int p = 0; p < P.np; ++p) {
                float *gc_ = B.g_pol[c][0] + p * plane + g;
                float *gq_ = B.g_pol[c][1] + p * plane + g;
                float gpc[4], gpp[4], c3[4];
                l4(gc_, gpc); l4(gq_, gpp); l4(P.c3[c] + p * plane + g, c3);
                const float c1 = P.c1[p], c2 = P.c2[p];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (!pv[q]) continue;
                    const float gE = ge[c][q];
                    const float gN = gpc[q] - gE / ec[q];
                    pe[c][q] += c3[q] * gN;
                    gpc[q] = d1[c][q] * gE / ec[q] + c1 * gN + gpp[q];
                    gpp[q] = c2 * gN;
                }
                s4(gc_, gpc); s4(gq_, gpp);
            }
        }
    }
    // PMC walls (core/stepper_3d.py _term_pmc :99-121): the tangential E on the wall is
    // live, and there the term differentiating along the wall's axis is zero
    const bool iL = iin || (P.pmc & 1), jL = jin || (P.pmc & 2);
    // E-side profiles (1, 0) on inert nodes
    const float exb = prof(P.pb[0][1], iin, 1.f, i), exa = prof(P.pa[0][1], iin, 0.f, i);
    const float eyb = prof(P.pb[1][1], jin, 1.f, j), eya = prof(P.pa[1][1], jin, 0.f, j);
    float t[9][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = kb + q;
        const bool vzE = k < nz, vz = k <= nz - 2, kin = k >= 1 && k <= nz - 2;
        const bool kL = kin || (P.pmc & 4);
        const float ezb = prof(P.pb[2][1], kin, 1.f, k), eza = prof(P.pa[2][1], kin, 0.f, k);
        // Ex: valid i <= nx-2, k < nz; curl on j, k interior
        {
            const bool v = xok && vzE, in = v && jL && kL;
            const float e_x = 0.5f * (ep[q] + epi[q]);
            const float gE = ge[0][q];
            t[6][q] = v ? -gE * (en[0][q] - d1[0][q] * eo[0][q]) / e_x : 0.f;
            const float gc = in ? d2[0][q] * gE / e_x : 0.f;
            ge[0][q] = v ? d1[0][q] * gE + pe[0][q] : gE;   // d1 gE (+ poles) to E
            const float g6 = gp[0][q] + gc, g7 = gp[1][q] - gc;
            const bool u6 = v && jin, u7 = v && kin;
            gp[0][q] = u6 ? eyb * g6 : gp[0][q];
            gp[1][q] = u7 ? ezb * g7 : gp[1][q];
            t[0][q] = u6 ? gc + eya * g6 : 0.f;                    // dy(Hz)
            t[1][q] = u7 ? -gc + eza * g7 : 0.f;                   // dz(Hy)
        }
        // Ey: valid j <= ny-2, k < nz; curl on i, k interior
        {
            const bool v = vyH && vzE, in = v && iL && kL;
            const float e_y = 0.5f * (ep[q] + epj[q]);
            const float gE = ge[1][q];
            t[7][q] = v ? -gE * (en[1][q] - d1[1][q] * eo[1][q]) / e_y : 0.f;
            const float gc = in ? d2[1][q] * gE / e_y : 0.f;
            ge[1][q] = v ? d1[1][q] * gE + pe[1][q] : gE;   // d1 gE (+ poles) to E
            const float g8 = gp[2][q] + gc, g9 = gp[3][q] - gc;
            const bool u8 = v && kin, u9 = v && iin;
            gp[2][q] = u8 ? ezb * g8 : gp[2][q];
            gp[3][q] = u9 ? exb * g9 : gp[3][q];
            t[2][q] = u8 ? gc + eza * g8 : 0.f;                    // dz(Hx)
            t[3][q] = u9 ? -gc + exa * g9 : 0.f;                   // dx(Hz)
        }
        // Ez: valid k <= nz-2; curl on i, j interior
        {
            const bool v = vz, in = v && iL && jL;
            const float e_z = 0.5f * (ep[q] + ((q < 3) ? ep[q + 1] : epk));
            const float gE = ge[2][q];
            t[8][q] = v ? -gE * (en[2][q] - d1[2][q] * eo[2][q]) / e_z : 0.f;
            const float gc = in ? d2[2][q] * gE / e_z : 0.f;
            ge[2][q] = v ? d1[2][q] * gE + pe[2][q] : gE;   // d1 gE (+ poles) to E
            const float g10 = gp[4][q] + gc, g11 = gp[5][q] - gc;
            const bool u10 = v && iin, u11 = v && jin;
            gp[4][q] = u10 ? exb * g10 : gp[4][q];
            gp[5][q] = u11 ? eyb * g11 : gp[5][q];
            t[4][q] = u10 ? gc + exa * g10 : 0.f;                  // dx(Hy)
            t[5][q] = u11 ? -gc + eya * g11 : 0.f;                 // dy(Hx)
        }
    }
    for (int c = 0; c < 6; ++c) s4(B.g_psi[6 + c] + g, gp[c]);
    for (int c = 0; c < 9; ++c) s4(B.tmp[c] + g, t[c]);
    if (damp || P.np > 0)
        for (int c = 0; c < 3; ++c) s4(B.g[c] + g, ge[c]);
}

__global__ void __launch_bounds__(32 * A3Y) k_adj3_h(const __grid_constant__ Adj3 P) {
    const int nx = P.nx, ny = P.ny, nz = P.nz, ZP = P.zp;
    const int lane = threadIdx.x;
    const int j = blockIdx.y * A3Y + threadIdx.y;
    const int i = blockIdx.z;
    const int kb = blockIdx.x * 128 + 4 * lane;
    const bool act = j < ny && kb < ZP;
    const uint32_t NYZ = (uint32_t)ny * ZP;
    const uint32_t g = (uint32_t)i * NYZ + (uint32_t)(j * ZP + kb);
    const mtb_adj3d_buffers &B = P.b;
    const float dt = P.dt, rdx = P.rdx;
    // own and +1 neighbours of the E-kernel adjoints
    float t0[4], t0j[4], t3[4], t3i[4], t1[4], t4[4], t4i[4], t2[4], t5[4], t5j[4];
    float t1k = 0.f, t2k = 0.f;
    zz(t0); zz(t0j); zz(t3); zz(t3i); zz(t1); zz(t4); zz(t4i); zz(t2); zz(t5); zz(t5j);
    if (act) {
        l4(B.tmp[0] + g, t0); l4(B.tmp[1] + g, t1); l4(B.tmp[2] + g, t2);
        l4(B.tmp[3] + g, t3); l4(B.tmp[4] + g, t4); l4(B.tmp[5] + g, t5);
        if (j + 1 < ny) { l4(B.tmp[0] + g + ZP, t0j); l4(B.tmp[5] + g + ZP, t5j); }
        if (i + 1 < nx) { l4(B.tmp[3] + g + NYZ, t3i); l4(B.tmp[4] + g + NYZ, t4i); }
        if (lane == 31 && kb + 4 < ZP) { t1k = B.tmp[1][g + 4]; t2k = B.tmp[2][g + 4]; }
    }
    {
        const float a = __shfl_down_sync(0xffffffffu, t1[0], 1);
        const float b = __shfl_down_sync(0xffffffffu, t2[0], 1);
        if (lane != 31) { t1k = a; t2k = b; }
    }
    if (!act) return;
    const bool xok = i <= nx - 2, vyH = j <= ny - 2;
    float gh[3][4], gp[6][4];
    for (int c = 0; c < 3; ++c) l4(B.g[3 + c] + g, gh[c]);
    for (int c = 0; c < 6; ++c) l4(B.g_psi[c] + g, gp[c]);
    const float hxb = prof(P.pb[0][0], xok, 1.f, i), hxa = prof(P.pa[0][0], xok, 0.f, i);
    const float hyb = prof(P.pb[1][0], vyH, 1.f, j), hya = prof(P.pa[1][0], vyH, 0.f, j);
    // conductive damping: H' = d1 H - d2 curl (core/stepper_3d.py:375-393)
    float h1[3][4], h2[3][4];
    for (int c = 0; c < 3; ++c)
        for (int q = 0; q < 4; ++q) { h1[c][q] = 1.f; h2[c][q] = dt; }
    if (P.dmp[3][0])
        for (int c = 0; c < 3; ++c) { l4(P.dmp[3 + c][0] + g, h1[c]); l4(P.dmp[3 + c][1] + g, h2[c]); }
    float u[6][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = kb + q;
        const bool vz = k <= nz - 2, vzE = k < nz;
        const float hzb = prof(P.pb[2][0], vz, 1.f, k), hza = prof(P.pa[2][0], vz, 0.f, k);
        const float t1n = (q < 3) ? t1[q + 1] : t1k;
        const float t2n = (q < 3) ? t2[q + 1] : t2k;
        // transposed differences of the E kernel's H derivatives
        const float gx = gh[0][q] + (t2[q] - t2n) * rdx + (t5[q] - t5j[q]) * rdx;
        const float gy = gh[1][q] + (t1[q] - t1n) * rdx + (t4[q] - t4i[q]) * rdx;
        const float gz = gh[2][q] + (t0[q] - t0j[q]) * rdx + (t3[q] - t3i[q]) * rdx;
        // Hx -= dt ((dy + psi0') - (dz + psi1')): valid j <= ny-2, k <= nz-2
        {
            const bool v = vyH && vz;
            const float c0 = -h2[0][q] * gx, c1 = h2[0][q] * gx;
            const float g0 = gp[0][q] + c0, g1 = gp[1][q] + c1;
            u[0][q] = v ? c0 + hya * g0 : 0.f;                     // dy(Ez)
            u[1][q] = v ? c1 + hza * g1 : 0.f;                     // dz(Ey)
            gp[0][q] = v ? hyb * g0 : gp[0][q];
            gp[1][q] = v ? hzb * g1 : gp[1][q];
            gh[0][q] = v ? h1[0][q] * gx : gx;
        }
        // Hy -= dt ((dz + psi2') - (dx + psi3')): valid i <= nx-2, k <= nz-2
        {
            const bool v = xok && vz;
            const float c2 = -h2[1][q] * gy, c3 = h2[1][q] * gy;
            const float g2 = gp[2][q] + c2, g3 = gp[3][q] + c3;
            u[2][q] = v ? c2 + hza * g2 : 0.f;                     // dz(Ex)
            u[3][q] = v ? c3 + hxa * g3 : 0.f;                     // dx(Ez)
            gp[2][q] = v ? hzb * g2 : gp[2][q];
            gp[3][q] = v ? hxb * g3 : gp[3][q];
            gh[1][q] = v ? h1[1][q] * gy : gy;
        }
        // Hz -= dt ((dx + psi4') - (dy + psi5')): valid i <= nx-2, j <= ny-2, k < nz
        {
            const bool v = xok && vyH && vzE;
            const float c4 = -h2[2][q] * gz, c5 = h2[2][q] * gz;
            const float g4 = gp[4][q] + c4, g5 = gp[5][q] + c5;
            u[4][q] = v ? c4 + hxa * g4 : 0.f;                     // dx(Ey)
            u[5][q] = v ? c5 + hya * g5 : 0.f;                     // dy(Ex)
            gp[4][q] = v ? hxb * g4 : gp[4][q];
            gp[5][q] = v ? hyb * g5 : gp[5][q];
            gh[2][q] = v ? h1[2][q] * gz : gz;
        }
    }
    for (int c = 0; c < 3; ++c) s4(B.g[3 + c] + g, gh[c]);
    for (int c = 0; c < 6; ++c) s4(B.g_psi[c] + g, gp[c]);
    for (int c = 0; c < 6; ++c) s4(B.tmp[9 + c] + g, u[c]);
}

__global__ void __launch_bounds__(32 * A3Y) k_adj3_fin(const __grid_constant__ Adj3 P) {
    const int nx = P.nx, ny = P.ny, nz = P.nz, ZP = P.zp;
    const int lane = threadIdx.x;
    const int j = blockIdx.y * A3Y + threadIdx.y;
    const int i = blockIdx.z;
    const int kb = blockIdx.x * 128 + 4 * lane;
    const bool act = j < ny && kb < ZP;
    const uint32_t NYZ = (uint32_t)ny * ZP;
    const uint32_t g = (uint32_t)i * NYZ + (uint32_t)(j * ZP + kb);
    const mtb_adj3d_buffers &B = P.b;
    const float rdx = P.rdx;
    // own and -1 neighbours of the H-kernel adjoints and of the eps parts
    float u9[4], u9j[4], u10[4], u11[4], u12[4], u12i[4], u13[4], u13i[4], u14[4], u14j[4];
    float t6[4], t6i[4], t7[4], t7j[4], t8[4];
    float u10k = 0.f, u11k = 0.f, t8k = 0.f;
    zz(u9); zz(u9j); zz(u10); zz(u11); zz(u12); zz(u12i); zz(u13); zz(u13i); zz(u14); zz(u14j);
    zz(t6); zz(t6i); zz(t7); zz(t7j); zz(t8);
    if (act) {
        l4(B.tmp[9] + g, u9); l4(B.tmp[10] + g, u10); l4(B.tmp[11] + g, u11);
        l4(B.tmp[12] + g, u12); l4(B.tmp[13] + g, u13); l4(B.tmp[14] + g, u14);
        l4(B.tmp[6] + g, t6); l4(B.tmp[7] + g, t7); l4(B.tmp[8] + g, t8);
        if (j >= 1) { l4(B.tmp[9] + g - ZP, u9j); l4(B.tmp[14] + g - ZP, u14j); l4(B.tmp[7] + g - ZP, t7j); }
        if (i >= 1) { l4(B.tmp[12] + g - NYZ, u12i); l4(B.tmp[13] + g - NYZ, u13i); l4(B.tmp[6] + g - NYZ, t6i); }
        if (lane == 0 && kb >= 1) { u10k = B.tmp[10][g - 1]; u11k = B.tmp[11][g - 1]; t8k = B.tmp[8][g - 1]; }
    }
    {
        const float a = __shfl_up_sync(0xffffffffu, u10[3], 1);
        const float b = __shfl_up_sync(0xffffffffu, u11[3], 1);
        const float c = __shfl_up_sync(0xffffffffu, t8[3], 1);
        if (lane != 0) { u10k = a; u11k = b; t8k = c; }
    }
    if (!act) return;
    float ge[3][4], geps[4];
    for (int c = 0; c < 3; ++c) l4(B.g[c] + g, ge[c]);
    l4(B.g_eps + g, geps);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = kb + q;
        const float u10m = (q == 0) ? u10k : u10[q - 1];
        const float u11m = (q == 0) ? u11k : u11[q - 1];
        const float t8m = (q == 0) ? t8k : t8[q - 1];
        // Ex: in dz(Ex) of Hy (k+1 - k) and dy(Ex) of Hz (j+1 - j)
        ge[0][q] += (u11m - u11[q]) * rdx + (u14j[q] - u14[q]) * rdx;
        // Ey: in dz(Ey) of Hx and dx(Ey) of Hz
        ge[1][q] += (u10m - u10[q]) * rdx + (u13i[q] - u13[q]) * rdx;
        // Ez: in dy(Ez) of Hx and dx(Ez) of Hy
        ge[2][q] += (u9j[q] - u9[q]) * rdx + (u12i[q] - u12[q]) * rdx;
        if (k < nz)
            geps[q] += 0.5f * (t6[q] + t6i[q]) + 0.5f * (t7[q] + t7j[q]) + 0.5f * (t8[q] + t8m);
    }
    for (int c = 0; c < 3; ++c) s4(B.g[c] + g, ge[c]);
    s4(B.g_eps + g, geps);
}

}  // namespace mtb

using namespace mtb;

struct mtb_yee3d_adjoint {
    mtb_yee3d_struct s{};
    Adj3 a{};
    DftState dft;
    DevBuf s_d, pstart_d;
    int n_planes = 0;
    int64_t n_samples = 0;
    int64_t last_launches = 0;
};

extern "C" {

int mtb_yee3d_adjoint_create(const mtb_yee3d_struct *s, const mtb_adj3d_buffers *bufs,
                             const mtb_dft_region *regions, int32_t n_regions,
                             const mtb_phase_group *groups, int32_t n_groups,
                             int64_t ring_slot_elems, int32_t ring_slots,
                             mtb_yee3d_adjoint **out) {
    if (!out || !s || !bufs) return fail(MTB_INVALID_ARG, "null argument");
    *out = nullptr;
    const mtb_yee3d_struct &S = *s;
    const bool dmp = S.damp[0][0] != nullptr;
    for (int c = 0; c < 6; ++c)
        for (int h = 0; h < 2; ++h)
            if ((S.damp[c][h] != nullptr) != dmp ||
                (S.damp[c][h] && (reinterpret_cast<uintptr_t>(S.damp[c][h]) & 15)))
                return fail(MTB_INVALID_ARG, "3D adjoint: damping needs all twelve arrays, "
                            "16-byte aligned");
    if (S.n_poles < 0 || S.n_poles > MTB_MAX_POLES)
        return fail(MTB_INVALID_ARG, "3D adjoint: n_poles %d", S.n_poles);
    if (S.pmc_axes & ~7) return fail(MTB_INVALID_ARG, "3D adjoint: pmc_axes %d", S.pmc_axes);
    if (S.nx < 3 || S.ny < 3 || S.nz < 3 || S.zpitch < S.nz || (S.zpitch & 3))
        return fail(MTB_INVALID_ARG, "3D adjoint: bad grid");
    if ((int64_t)S.nx * S.ny * S.zpitch >= (1LL << 31) || S.nx > 65535 ||
        (S.ny + A3Y - 1) / A3Y > 65535)
        return fail(MTB_UNSUPPORTED, "3D adjoint: grid too large");
    auto bad = [](const void *p) { return !p || (reinterpret_cast<uintptr_t>(p) & 15); };
    for (int c = 0; c < 6; ++c)
        if (bad(bufs->g[c])) return fail(MTB_INVALID_ARG, "3D adjoint: bad g buffer");
    for (int c = 0; c < 12; ++c)
        if (bad(bufs->g_psi[c])) return fail(MTB_INVALID_ARG, "3D adjoint: bad g_psi buffer");
    for (int c = 0; c < 15; ++c)
        if (bad(bufs->tmp[c])) return fail(MTB_INVALID_ARG, "3D adjoint: bad tmp buffer");
    if (bad(bufs->g_eps) || bad(S.eps)) return fail(MTB_INVALID_ARG, "3D adjoint: bad eps");
    if (S.n_poles > 0)
        for (int c = 0; c < 3; ++c)
            if (bad(S.pol_c3[c]) || bad(bufs->g_pol[c][0]) || bad(bufs->g_pol[c][1]))
                return fail(MTB_INVALID_ARG, "3D adjoint: poles need c3 and both g_pol stacks "
                            "per component, 16-byte aligned");
    for (int a = 0; a < 3; ++a)
        for (int h = 0; h < 2; ++h)
            if (!S.prof_b[a][h] || !S.prof_a[a][h])
                return fail(MTB_INVALID_ARG, "3D adjoint: null CPML profile");
    if (S.n_planes < 0 || (S.n_planes > 0 && (!S.planes || !S.plane_ring_off)))
        return fail(MTB_INVALID_ARG, "3D adjoint: bad plane list");
    mtb_yee3d_adjoint *p = new mtb_yee3d_adjoint();
    p->s = S;
    Adj3 &A = p->a;
    A.b = *bufs;
    A.eps = S.eps;
    for (int a = 0; a < 3; ++a)
        for (int h = 0; h < 2; ++h) {
            A.pb[a][h] = S.prof_b[a][h];
            A.pa[a][h] = S.prof_a[a][h];
        }
    for (int c = 0; c < 6; ++c)
        for (int h = 0; h < 2; ++h) A.dmp[c][h] = S.damp[c][h];
    A.np = S.n_poles;
    A.pmc = S.pmc_axes;
    for (int c = 0; c < 3; ++c) A.c3[c] = S.n_poles ? S.pol_c3[c] : nullptr;
    for (int p = 0; p < MTB_MAX_POLES; ++p) {
        A.c1[p] = p < S.n_poles ? S.pol_c1[p] : 0.f;
        A.c2[p] = p < S.n_poles ? S.pol_c2[p] : 0.f;
    }
    A.nx = S.nx; A.ny = S.ny; A.nz = S.nz; A.zp = S.zpitch;
    A.dt = S.dt;
    A.rdx = 1.0f / S.dx;
    int rc = p->dft.init(regions, n_regions, groups, n_groups, ring_slot_elems,
                         ring_slots > 0 ? ring_slots : 32);
    if (!rc) rc = p->s_d.ensure(sizeof(mtb_yee3d_struct));
    if (!rc) rc = p->pstart_d.ensure(sizeof(int64_t) * (S.n_planes + 1));
    if (!rc && n_regions == 0)
        rc = p->dft.ring_d.ensure(sizeof(float) * (size_t)std::max<int64_t>(ring_slot_elems, 4) *
                                  p->dft.slots);
    if (rc) { p->dft.release(); delete p; return rc; }
    std::vector<int64_t> ps(S.n_planes + 1, 0);
    if (S.n_planes > 0) {
        std::vector<int32_t> pl(8 * S.n_planes);
        cudaError_t e = cudaMemcpy(pl.data(), S.planes, sizeof(int32_t) * 8 * S.n_planes,
                                   cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            p->dft.release(); delete p;
            return fail(MTB_CUDA_ERROR, "reading plane list: %s", cudaGetErrorString(e));
        }
        for (int q = 0; q < S.n_planes; ++q)
            ps[q + 1] = ps[q] + (int64_t)(pl[8 * q + 4] - pl[8 * q + 3]) *
                                    (pl[8 * q + 6] - pl[8 * q + 5]);
    }
    p->n_planes = S.n_planes;
    p->n_samples = ps[S.n_planes];
    cudaError_t e = cudaMemcpy(p->s_d.p, &S, sizeof(S), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(p->pstart_d.p, ps.data(), sizeof(int64_t) * ps.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        p->dft.release(); delete p;
        return fail(MTB_CUDA_ERROR, "3D adjoint upload: %s", cudaGetErrorString(e));
    }
    *out = p;
    return MTB_OK;
}

int mtb_yee3d_adjoint_run(mtb_yee3d_adjoint *p, int64_t t0, int32_t k, const float *rec,
                          int64_t rec_comp_stride, int64_t rec_slot_stride, void *stream) {
    if (!p) return fail(MTB_INVALID_ARG, "3D adjoint plan is null");
    p->last_launches = 0;
    if (k <= 0) return MTB_OK;
    if (k > p->dft.slots) return fail(MTB_INVALID_ARG, "k %d > ring slots %d", k, p->dft.slots);
    if (!rec || (reinterpret_cast<uintptr_t>(rec) & 15) || (rec_comp_stride & 3) ||
        (rec_slot_stride & 3))
        return fail(MTB_INVALID_ARG, "3D adjoint: bad forward record");
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    if ((rc = p->dft.upload_phases(t0, k, st))) return rc;
    if (p->dft.n_regions > 0) {
        if ((rc = p->dft.expand(0, k, st))) return rc;
        ++p->last_launches;
    } else {
        MTB_CUDA_TRY(cudaMemsetAsync(p->dft.ring_d.p, 0,
                                     sizeof(float) * (size_t)p->dft.slot_elems * k, st));
    }
    const Adj3 &A = p->a;
    const dim3 blk(32, A3Y);
    const dim3 grid((A.zp + 127) / 128, (A.ny + A3Y - 1) / A3Y, A.nx);
    for (int q = k - 1; q >= 0; --q) {
        const float *radj = p->dft.ring_d.as<float>() + (size_t)q * p->dft.slot_elems;
        if (p->n_samples > 0) {
            k_adj3_inject<<<(unsigned)((p->n_samples + 255) / 256), 256, 0, st>>>(
                p->s_d.as<mtb_yee3d_struct>(), p->pstart_d.as<int64_t>(), p->n_planes, radj, A.b);
            MTB_CHECK_LAUNCH();
            ++p->last_launches;
        }
        const float *en = rec + (size_t)(q + 1) * rec_slot_stride;
        const float *eo = rec + (size_t)q * rec_slot_stride;
        k_adj3_e<<<grid, blk, 0, st>>>(A, en, eo, rec_comp_stride);
        MTB_CHECK_LAUNCH();
        k_adj3_h<<<grid, blk, 0, st>>>(A);
        MTB_CHECK_LAUNCH();
        k_adj3_fin<<<grid, blk, 0, st>>>(A);
        MTB_CHECK_LAUNCH();
        p->last_launches += 3;
    }
    return MTB_OK;
}

int64_t mtb_yee3d_adjoint_last_launches(const mtb_yee3d_adjoint *p) {
    return p ? p->last_launches : -1;
}

void mtb_yee3d_adjoint_destroy(mtb_yee3d_adjoint *p) {
    if (!p) return;
    p->dft.release();
    p->s_d.release();
    p->pstart_d.release();
    delete p;
}

}  // extern "C"
