// 3D Yee step with CPML (the functional stepper's CPML path,
// core/stepper_3d.py:363-445, and its soft source :448-482) for sm_100a.
//
// A block owns TY consecutive y rows of one x segment and the whole z
// extent; warp (wy, wz) owns row j0+wy and z columns wz*128 + 4*lane .. +3
// (one float4 per array). The block marches along x. Per plane i:
//   A  E(n) of plane i for rows j0-1 .. j0+TY and eps(i) go to shared memory
//      (own rows from registers, the two halo rows loaded by halo warps);
//      every warp loads E(n) and eps of plane i+1 into registers.
//   B  __syncthreads
//   C  H(n+1/2) of plane i for rows j0-1 .. j0+TY-1 (row j0-1 is recomputed
//      by the halo warps and never stored) -> shared memory and HBM.
//   D  __syncthreads
//   E  E(n+1) of plane i for the own rows; source cells; store.
// E is stored (as in the functional stepper), eps is cell-centred and
// Yee-averaged in the kernel exactly as core/stepper_3d.py:_avg does.
// Evolving arrays are ping-pong pairs because of the halo recomputation.
#include <algorithm>
#include <mutex>
#include <vector>

#include <cudaTypedefs.h>

#include "mtb_common.cuh"

namespace mtb {

constexpr int TY3 = 4;          // own rows per block
constexpr int MAXNZ = 4;        // z warps per row (zpitch <= 512)

struct Ctx3D {
    const float *amp;           // coefficient of this step
    int par;
};

__device__ __forceinline__ void ld4v(const float *p, float (&v)[4]) {
    const float4 x = *reinterpret_cast<const float4 *>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void st4v(float *p, const float (&v)[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void z4(float (&v)[4]) { v[0] = v[1] = v[2] = v[3] = 0.f; }

// profile activity (psi is touched only where the layer is active)
__device__ __forceinline__ bool pact(float b, float a) { return a != 0.f || b != 1.f; }

template <int NZW>
__global__ void __launch_bounds__(32 * NZW * (TY3 + 2)) k_yee3d_step(
    const mtb_yee3d_struct *__restrict__ SS, int rows_per_seg, Ctx3D C) {
    const mtb_yee3d_struct &S = *SS;
    const int nx = S.nx, ny = S.ny, nz = S.nz;
    const int ZP = S.zpitch;
    const int ZS = ZP + 4;                       // shared row stride (floats)
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wy = warp / NZW, wz = warp % NZW;
    const int j0 = blockIdx.x * TY3;
    const int i0 = blockIdx.y * rows_per_seg;
    const int i1 = min(i0 + rows_per_seg, nx);
    const int kb = wz * 128 + 4 * lane;
    const bool kact = kb < ZP;
    // role: own row, H halo row (j0-1) or E halo row (j0+TY)
    const bool own = wy < TY3;
    const bool hhalo = wy == TY3;
    const bool ehalo = wy == TY3 + 1;
    const int j = own ? j0 + wy : (hhalo ? j0 - 1 : j0 + TY3);
    const bool jok = j >= 0 && j < ny;
    const bool act = kact && jok;
    const int sr = own ? wy + 1 : (hhalo ? 0 : TY3 + 1);   // shared row of j
    const float dt = S.dt, rdx = 1.0f / S.dx;
    const int par = C.par;
    const int64_t NYZ = (int64_t)ny * ZP;
    auto gidx = [&](int i, int jj) -> int64_t { return (int64_t)i * NYZ + (int64_t)jj * ZP + kb; };

    extern __shared__ float sm[];
    // E(n) plane i, rows j0-1 .. j0+TY: sE[c][row][z]; eps(i) sEp[row][z]
    float *sE = sm;
    float *sEp = sE + 3 * (TY3 + 2) * ZS;
    // H(n+1/2) plane i, rows j0-1 .. j0+TY-1: sH[c][row][z]
    float *sH = sEp + (TY3 + 2) * ZS;
    auto SE = [&](int c, int r) -> float * { return sE + (c * (TY3 + 2) + r) * ZS; };
    auto SH = [&](int c, int r) -> float * { return sH + (c * (TY3 + 1) + r) * ZS; };

    const float *Eo[3] = {S.f[0][par], S.f[1][par], S.f[2][par]};
    float *En[3] = {S.f[0][par ^ 1], S.f[1][par ^ 1], S.f[2][par ^ 1]};
    const float *Ho[3] = {S.f[3][par], S.f[4][par], S.f[5][par]};
    float *Hn[3] = {S.f[3][par ^ 1], S.f[4][par ^ 1], S.f[5][par ^ 1]};
    const float *eps = S.eps;

    // lane-constant z profiles (half nodes for H, integer nodes for E)
    bool vzH[4], vzE[4], hzA[4], ezA[4], kin[4];
    float hzb[4], hza[4], ezb[4], eza[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = kb + q;
        vzH[q] = k <= nz - 2;
        vzE[q] = k < nz;
        kin[q] = k >= 1 && k <= nz - 2;
        hzb[q] = vzH[q] ? __ldg(S.prof_b[2][0] + k) : 1.f;
        hza[q] = vzH[q] ? __ldg(S.prof_a[2][0] + k) : 0.f;
        ezb[q] = vzE[q] ? __ldg(S.prof_b[2][1] + k) : 1.f;
        eza[q] = vzE[q] ? __ldg(S.prof_a[2][1] + k) : 0.f;
        hzA[q] = vzH[q] && pact(hzb[q], hza[q]);
        ezA[q] = kin[q] && pact(ezb[q], eza[q]);
    }
    const bool anyHz = act && (hzA[0] || hzA[1] || hzA[2] || hzA[3]);
    const bool anyEz = act && (ezA[0] || ezA[1] || ezA[2] || ezA[3]);
    // row-uniform y profiles
    const bool vyH = j >= 0 && j <= ny - 2;
    const bool jin = j >= 1 && j <= ny - 2;
    float hyb = 1.f, hya = 0.f, eyb = 1.f, eya = 0.f;
    if (vyH) { hyb = __ldg(S.prof_b[1][0] + j); hya = __ldg(S.prof_a[1][0] + j); }
    if (jok) { eyb = __ldg(S.prof_b[1][1] + j); eya = __ldg(S.prof_a[1][1] + j); }
    const bool hyA = act && vyH && pact(hyb, hya);
    const bool eyA = act && jin && pact(eyb, eya);
    const int kl = wz * 128 + 128;               // first column of the next z warp

    float e1[3][4], ep1[4];                       // E(n), eps of plane i+1 (registers)
    float hyP[4], hzP[4];                         // H(n+1/2) of plane i-1 (own rows)
    z4(hyP); z4(hzP);

    auto load_plane = [&](int i, float (&e)[3][4], float (&ep)[4]) {
        if (act && i >= 0 && i < nx) {
            const int64_t g = gidx(i, j);
            ld4v(Eo[0] + g, e[0]); ld4v(Eo[1] + g, e[1]); ld4v(Eo[2] + g, e[2]);
            const float4 x = __ldg(reinterpret_cast<const float4 *>(eps + g));
            ep[0] = x.x; ep[1] = x.y; ep[2] = x.z; ep[3] = x.w;
        } else {
            z4(e[0]); z4(e[1]); z4(e[2]);
            ep[0] = ep[1] = ep[2] = ep[3] = 1.f;
        }
    };

    const int ifirst = (i0 > 0) ? i0 - 1 : i0;
    {   // E(n) of plane ifirst into registers (becomes "plane i" at the first A)
        load_plane(ifirst, e1, ep1);
    }
    for (int i = ifirst; i < i1; ++i) {
        const bool work = i >= i0;               // plane i0-1 only prepares H(i0-1)
        // ---- A: publish E(n), eps of plane i; fetch plane i+1
        if (kact) {
            st4v(SE(0, sr) + kb, e1[0]);
            st4v(SE(1, sr) + kb, e1[1]);
            st4v(SE(2, sr) + kb, e1[2]);
            st4v(sEp + sr * ZS + kb, ep1);
        }
        float ec[3][4], epc[4];                   // E(n), eps of plane i (own)
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int q = 0; q < 4; ++q) ec[c][q] = e1[c][q];
#pragma unroll
        for (int q = 0; q < 4; ++q) epc[q] = ep1[q];
        if (!ehalo) load_plane(i + 1, e1, ep1);
        else { z4(e1[0]); z4(e1[1]); z4(e1[2]); ep1[0] = ep1[1] = ep1[2] = ep1[3] = 1.f; }
        __syncthreads();
        if (ehalo) {   // the E-halo warps only load the next plane for the next A
            if (i + 1 < i1) load_plane(i + 1, e1, ep1);
        }

        // ---- C: H(n+1/2) of plane i, rows j (own and H-halo)
        // eps neighbours for step E's Yee averages, eps(i, j+1) and
        // eps(i, k+1), are read here: the next plane's step A overwrites sEp
        // and no barrier separates it from this plane's step E.
        float epj1[4];
        if (kact && !ehalo) ld4v(sEp + (sr + 1) * ZS + kb, epj1); else z4(epj1);
        float epk1 = __shfl_down_sync(0xffffffffu, epc[0], 1);
        if (lane == 31) epk1 = (kl < ZP && !ehalo) ? sEp[sr * ZS + kl] : 1.f;
        float hn[3][4];
        if (!ehalo) {
            const bool xok = i <= nx - 2;
            float hxb = 1.f, hxa = 0.f;
            if (xok) { hxb = __ldg(S.prof_b[0][0] + i); hxa = __ldg(S.prof_a[0][0] + i); }
            const bool hxA = act && xok && pact(hxb, hxa);
            // neighbours: E(j+1) row, E(k+1) column
            float ezj1[4], exj1[4];
            if (kact) { ld4v(SE(2, sr + 1) + kb, ezj1); ld4v(SE(0, sr + 1) + kb, exj1); }
            else { z4(ezj1); z4(exj1); }
            float eyk1 = __shfl_down_sync(0xffffffffu, ec[1][0], 1);
            float exk1 = __shfl_down_sync(0xffffffffu, ec[0][0], 1);
            if (lane == 31) {
                eyk1 = (kl < ZP) ? SE(1, sr)[kl] : 0.f;
                exk1 = (kl < ZP) ? SE(0, sr)[kl] : 0.f;
            }
            const int64_t g = act ? gidx(i, j) : 0;
            const bool store = own && work && act;
            // Hx (core/stepper_3d.py:368-375): valid j <= ny-2, k <= nz-2
            {
                float h[4], pY[4], pZ[4];
                if (act) ld4v(Ho[0] + g, h); else z4(h);
                if (hyA) ld4v(S.psi[0][par] + g, pY); else z4(pY);
                if (anyHz && vyH) ld4v(S.psi[1][par] + g, pZ); else z4(pZ);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (!(vyH && vzH[q])) continue;
                    const float eyn = (q < 3) ? ec[1][q + 1] : eyk1;
                    const float dy = (ezj1[q] - ec[2][q]) * rdx;
                    const float dz = (eyn - ec[1][q]) * rdx;
                    float cy = dy, cz = dz;
                    if (hyA) { pY[q] = hyb * pY[q] + hya * dy; cy = dy + pY[q]; }
                    if (hzA[q]) { pZ[q] = hzb[q] * pZ[q] + hza[q] * dz; cz = dz + pZ[q]; }
                    h[q] = h[q] - dt * (cy - cz);
                }
                if (store) {
                    st4v(Hn[0] + g, h);
                    if (hyA) st4v(S.psi[0][par ^ 1] + g, pY);
                    if (anyHz && vyH) st4v(S.psi[1][par ^ 1] + g, pZ);
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) hn[0][q] = h[q];
            }
            // Hy (core/stepper_3d.py:377-384): valid i <= nx-2, k <= nz-2
            {
                float h[4], pZ[4], pX[4];
                if (act) ld4v(Ho[1] + g, h); else z4(h);
                if (anyHz && xok) ld4v(S.psi[2][par] + g, pZ); else z4(pZ);
                if (hxA) ld4v(S.psi[3][par] + g, pX); else z4(pX);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (!(xok && vzH[q])) continue;
                    const float exn = (q < 3) ? ec[0][q + 1] : exk1;
                    const float dz = (exn - ec[0][q]) * rdx;
                    const float dx = (e1[2][q] - ec[2][q]) * rdx;
                    float cz = dz, cx = dx;
                    if (hzA[q]) { pZ[q] = hzb[q] * pZ[q] + hza[q] * dz; cz = dz + pZ[q]; }
                    if (hxA) { pX[q] = hxb * pX[q] + hxa * dx; cx = dx + pX[q]; }
                    h[q] = h[q] - dt * (cz - cx);
                }
                if (store) {
                    st4v(Hn[1] + g, h);
                    if (anyHz && xok) st4v(S.psi[2][par ^ 1] + g, pZ);
                    if (hxA) st4v(S.psi[3][par ^ 1] + g, pX);
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) hn[1][q] = h[q];
            }
            // Hz (core/stepper_3d.py:386-393): valid i <= nx-2, j <= ny-2
            {
                float h[4], pX[4], pY[4];
                if (act) ld4v(Ho[2] + g, h); else z4(h);
                if (hxA && vyH) ld4v(S.psi[4][par] + g, pX); else z4(pX);
                if (hyA && xok) ld4v(S.psi[5][par] + g, pY); else z4(pY);
                if (xok && vyH) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        if (!vzE[q]) continue;
                        const float dx = (e1[1][q] - ec[1][q]) * rdx;
                        const float dy = (exj1[q] - ec[0][q]) * rdx;
                        float cx = dx, cy = dy;
                        if (hxA) { pX[q] = hxb * pX[q] + hxa * dx; cx = dx + pX[q]; }
                        if (hyA) { pY[q] = hyb * pY[q] + hya * dy; cy = dy + pY[q]; }
                        h[q] = h[q] - dt * (cx - cy);
                    }
                }
                if (store) {
                    st4v(Hn[2] + g, h);
                    if (hxA && vyH) st4v(S.psi[4][par ^ 1] + g, pX);
                    if (hyA && xok) st4v(S.psi[5][par ^ 1] + g, pY);
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) hn[2][q] = h[q];
            }
            if (kact) {
                const int hr = own ? wy + 1 : 0;
                st4v(SH(0, hr) + kb, hn[0]);
                st4v(SH(1, hr) + kb, hn[1]);
                st4v(SH(2, hr) + kb, hn[2]);
            }
        }
        __syncthreads();

        // ---- E: E(n+1) of plane i, own rows
        if (own && work) {
            const int hr = wy + 1;                      // shared H row of j; j-1 is hr-1
            const bool iin = i >= 1 && i <= nx - 2;
            float exb = 1.f, exa = 0.f;
            if (i < nx) { exb = __ldg(S.prof_b[0][1] + i); exa = __ldg(S.prof_a[0][1] + i); }
            const bool exA = act && iin && pact(exb, exa);
            float hzm[4], hxm[4];                       // H(j-1) rows
            if (kact) { ld4v(SH(2, hr - 1) + kb, hzm); ld4v(SH(0, hr - 1) + kb, hxm); }
            else { z4(hzm); z4(hxm); }
            float hyk = __shfl_up_sync(0xffffffffu, hn[1][3], 1);   // H(k-1)
            float hxk = __shfl_up_sync(0xffffffffu, hn[0][3], 1);
            if (lane == 0) {
                const int kk = wz * 128 - 1;
                hyk = (kk >= 0) ? SH(1, hr)[kk] : 0.f;
                hxk = (kk >= 0) ? SH(0, hr)[kk] : 0.f;
            }
            const int64_t g = act ? gidx(i, j) : 0;
            float en[3][4];
            // The psi recursions run over their own arrays' full extent
            // (core/stepper_3d.py:79-101 State3D shapes), wider than the
            // interior where the curl is applied (_pad_interior).
            // Ex (core/stepper_3d.py:397-409): valid i <= nx-2
            {
                float pY[4], pZ[4];
                const bool xok = i <= nx - 2;
                const bool ldY = eyA && xok, ldZ = anyEz && xok;
                if (ldY) ld4v(S.psi[6][par] + g, pY); else z4(pY);
                if (ldZ) ld4v(S.psi[7][par] + g, pZ); else z4(pZ);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float hym = (q == 0) ? hyk : hn[1][q - 1];
                    const float dy = (hn[2][q] - hzm[q]) * rdx;      // psi_Hz_y: j interior, all k
                    const float dz = (hn[1][q] - hym) * rdx;         // psi_Hy_z: k interior, all j
                    float cy = dy, cz = dz;
                    if (ldY && vzE[q]) { pY[q] = eyb * pY[q] + eya * dy; cy = dy + pY[q]; }
                    if (ldZ && ezA[q]) { pZ[q] = ezb[q] * pZ[q] + eza[q] * dz; cz = dz + pZ[q]; }
                    const float curl = (xok && jin && kin[q]) ? (cy - cz) : 0.f;
                    float v = ec[0][q];
                    if (xok && vzE[q] && act) {
                        const float e_x = 0.5f * (epc[q] + ep1[q]);
                        v = (v * e_x + dt * curl) / e_x;
                    }
                    en[0][q] = v;
                }
                if (ldY) st4v(S.psi[6][par ^ 1] + g, pY);
                if (ldZ) st4v(S.psi[7][par ^ 1] + g, pZ);
            }
            // Ey (core/stepper_3d.py:411-422): valid j <= ny-2
            {
                float pZ[4], pX[4];
                const bool ldZ = anyEz && vyH, ldX = exA && vyH;
                if (ldZ) ld4v(S.psi[8][par] + g, pZ); else z4(pZ);
                if (ldX) ld4v(S.psi[9][par] + g, pX); else z4(pX);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float hxkm = (q == 0) ? hxk : hn[0][q - 1];
                    const float dz = (hn[0][q] - hxkm) * rdx;        // psi_Hx_z: k interior, all i
                    const float dx = (hn[2][q] - hzP[q]) * rdx;      // psi_Hz_x: i interior, all k
                    float cz = dz, cx = dx;
                    if (ldZ && ezA[q]) { pZ[q] = ezb[q] * pZ[q] + eza[q] * dz; cz = dz + pZ[q]; }
                    if (ldX && vzE[q]) { pX[q] = exb * pX[q] + exa * dx; cx = dx + pX[q]; }
                    const float curl = (vyH && iin && kin[q]) ? (cz - cx) : 0.f;
                    float v = ec[1][q];
                    if (vyH && vzE[q] && act) {
                        const float e_y = 0.5f * (epc[q] + epj1[q]);
                        v = (v * e_y + dt * curl) / e_y;
                    }
                    en[1][q] = v;
                }
                if (ldZ) st4v(S.psi[8][par ^ 1] + g, pZ);
                if (ldX) st4v(S.psi[9][par ^ 1] + g, pX);
            }
            // Ez (core/stepper_3d.py:424-437): valid k <= nz-2
            {
                float pX[4], pY[4];
                const bool ldX = exA, ldY = eyA;
                if (ldX) ld4v(S.psi[10][par] + g, pX); else z4(pX);
                if (ldY) ld4v(S.psi[11][par] + g, pY); else z4(pY);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float dx = (hn[1][q] - hyP[q]) * rdx;      // psi_Hy_x: i interior, all j
                    const float dy = (hn[0][q] - hxm[q]) * rdx;      // psi_Hx_y: j interior, all i
                    float cx = dx, cy = dy;
                    if (ldX && vzH[q]) { pX[q] = exb * pX[q] + exa * dx; cx = dx + pX[q]; }
                    if (ldY && vzH[q]) { pY[q] = eyb * pY[q] + eya * dy; cy = dy + pY[q]; }
                    const float curl = (iin && jin && vzH[q]) ? (cx - cy) : 0.f;
                    float v = ec[2][q];
                    if (vzH[q] && act) {
                        const float e_z = 0.5f * (epc[q] + ((q < 3) ? epc[q + 1] : epk1));
                        v = (v * e_z + dt * curl) / e_z;
                    }
                    en[2][q] = v;
                }
                if (ldX) st4v(S.psi[10][par ^ 1] + g, pX);
                if (ldY) st4v(S.psi[11][par ^ 1] + g, pY);
            }
            // soft current cells of row (i, j) on component src_comp
            if (act && S.src.n > 0) {
                const int r = i * ny + j;
                const int e0 = __ldg(S.src.row_ptr + r), e1x = __ldg(S.src.row_ptr + r + 1);
                if (e0 < e1x) {
                    const int c = S.src_comp;
                    const float a = __ldg(C.amp + S.src.amp_col);
                    const float sgn = S.src_is_point ? (float)S.point_sign : -1.f;
                    for (int e = e0; e < e1x; ++e) {
                        const int kq = __ldg(S.src.col + e) - kb;
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            if (kq != q) continue;
                            float epc_ = epc[q];
                            float epn;
                            if (c == 0) epn = ep1[q];
                            else if (c == 1) epn = epj1[q];
                            else epn = (q < 3) ? epc[q + 1] : epk1;
                            const float ecomp = 0.5f * (epc_ + epn);
                            const float v = a * __ldg(S.src.w + e);
                            if (S.src_is_point) en[c][q] += sgn * (v * (1.0f / ecomp));
                            else en[c][q] -= v / ecomp;
                        }
                    }
                }
            }
            if (act) {
                st4v(En[0] + g, en[0]);
                st4v(En[1] + g, en[1]);
                st4v(En[2] + g, en[2]);
            }
        }
        if (own) {
#pragma unroll
            for (int q = 0; q < 4; ++q) { hyP[q] = hn[1][q]; hzP[q] = hn[2][q]; }
        }
    }
}

// ---------------------------------------------------------------- split H / E kernels
// Streaming variant: one kernel advances H, a second E. A thread updates one
// float4 of z (4 cells) of one (i, j) row; a block is 32 x 8 threads = 128 z
// x 8 y of one x plane. Neighbours in y and x come from L1/L2 (the blocks of
// planes i and i+1 run concurrently), z+-1 from a warp shuffle.
//  * Every load a thread needs is issued before the first use of any: the
//    CPML memory is gated by the plan's band limits (geometry), not by the
//    loaded profile values, so a cell costs one memory round trip.
//  * The arithmetic is uniform across lanes: outside the layers the CPML
//    terms run with (b, a) = (1, 0) on psi = 0, which is the reference's own
//    arithmetic there, and the edge rules are selects, so a warp that holds
//    both layer and interior cells does not diverge.
//  * All pointers of one parity are resolved on the host into a by-value
//    parameter block (no pointer loads in the kernel).
// DRAM traffic is ~76 B per cell and step plus the CPML memory in the layers.
constexpr int SPLIT_Y = 8;

// Index k of an axis lies in a CPML band iff k < lo or k >= hi. Superset of
// the profile's active nodes; psi is loaded / stored there and updated with
// the profile's (b, a), which are (1, 0) on inactive nodes.
// [axis][0 H-side, 1 E-side]
struct Band3 {
    int lo[3][2];
    int hi[3][2];
};
__device__ __forceinline__ bool inband(const Band3 &B, int a, int h, int k) {
    return k < B.lo[a][h] || k >= B.hi[a][h];
}

// Rounding of the 3D updates, written out (no multiply-add contraction is left to the
// compiler), so that the split kernels and both paths of the one-pass kernel round
// alike and agree bit for bit.
__device__ __forceinline__ float y3_d(float a, float b, float rdx) {      // (a - b) / dx
    return __fmul_rn(__fsub_rn(a, b), rdx);
}
// CPML-stretched derivative d + q with q = b psi + a d (kappa = 1); q is the new psi
__device__ __forceinline__ float y3_s(float d, float b, float a, float psi, float &q) {
    q = __fmaf_rn(b, psi, __fmul_rn(a, d));
    return __fadd_rn(d, q);
}
__device__ __forceinline__ float y3_ec(float e0, float e1) {            // Yee-averaged eps
    return __fmul_rn(0.5f, __fadd_rn(e0, e1));
}
// H' = H - dt curl; with damping d1 H - d2 curl
__device__ __forceinline__ float y3_h(float h, float cu, float dt) { return __fmaf_rn(-dt, cu, h); }
__device__ __forceinline__ float y3_hd(float h, float cu, float d1, float d2) {
    return __fmaf_rn(-d2, cu, __fmul_rn(d1, h));
}
// E' = E + dt curl / eps_c (fast divide); with damping d1 E + d2 curl / eps_c; with
// poles the folded-D forms E + (dt curl + sum P(n) - sum P(n+1)) / eps_c and
// (d1 (eps_c E + sum P(n)) + d2 curl - sum P(n+1)) / eps_c
__device__ __forceinline__ float y3_e(float e, float curl, float dt, float ec) {
    return __fadd_rn(e, __fdividef(__fmul_rn(dt, curl), ec));
}
__device__ __forceinline__ float y3_ed(float e, float curl, float d1, float d2, float ec) {
    return __fadd_rn(__fmul_rn(d1, e), __fdividef(__fmul_rn(d2, curl), ec));
}
__device__ __forceinline__ float y3_ep(float e, float curl, float dt, float ec, float spc,
                                       float spn) {
    return __fadd_rn(e, __fdividef(__fsub_rn(__fmaf_rn(dt, curl, spc), spn), ec));
}
__device__ __forceinline__ float y3_epd(float e, float curl, float d1, float d2, float ec,
                                        float spc, float spn) {
    return __fdividef(__fsub_rn(__fmaf_rn(d2, curl, __fmul_rn(d1, __fmaf_rn(e, ec, spc))), spn),
                      ec);
}
// One E-update curl ta - tb (core/stepper_3d.py:395-437 with _term_pmc / _pad_interior,
// :86-121): wa / wb mark a cell on a wall of the axis that term a / b differentiates
// along; on a PEC wall (pa / pb clear) the tangential E keeps its value (curl 0), on a
// PMC wall that term alone is zero. Without PMC this is (wa || wb) ? 0 : ta - tb.
__device__ __forceinline__ float y3_curl(float ta, bool wa, bool pa, float tb, bool wb, bool pb) {
    return ((wa && !pa) || (wb && !pb)) ? 0.f : __fsub_rn(wa ? 0.f : ta, wb ? 0.f : tb);
}
// soft current of one cell: E + sgn v / eps_c (point) or E - v / eps_c (area / plane)
__device__ __forceinline__ float y3_src(float e, float v, float ecomp, bool point, float sgn) {
    return point ? __fadd_rn(e, sgn * __fmul_rn(v, __fdiv_rn(1.0f, ecomp)))
                 : __fsub_rn(e, __fdiv_rn(v, ecomp));
}

// One parity's pointers and sizes for the split kernels.
struct Split3 {
    const float *e[3];          // E(n)
    float *eo[3];               // E(n+1)
    const float *h[3];          // H(n-1/2)
    float *ho[3];               // H(n+1/2): written by the H kernel, read by the E kernel
    const float *pi[12];        // psi in
    float *po[12];              // psi out
    const float *eps;
    const float *pb[3][2];      // CPML b, a: [axis][0 H-side (n-1 nodes), 1 E-side (n nodes)]
    const float *pa[3][2];
    const int32_t *src_row;
    const int32_t *src_col;
    const float *src_w;
    int src_n, src_comp, src_is_point, point_sign;
    int nx, ny, nz, zp;
    float dt, rdx;
    Band3 B;
    const float *dmp[6][2];     // conductive damping (d1, d2) per component, or null
    // dispersive poles: per E component a stack of np box planes (plane floats apart),
    // P ping-pong with the fields, c3 per cell, c1 / c2 per pole
    float *pp[3][2];
    const float *pc3[3];
    float pc1[MTB_MAX_POLES], pc2[MTB_MAX_POLES];
    int np;
    uint32_t plane;
    int pmc;                    // PMC wall axes: bit 0 x, 1 y, 2 z (PEC otherwise)
};

__device__ __forceinline__ void ldg4v(const float *p, float (&v)[4]) {
    const float4 x = __ldg(reinterpret_cast<const float4 *>(p));
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void one4(float (&v)[4]) { v[0] = v[1] = v[2] = v[3] = 1.f; }

// H(n+1/2) from E(n): core/stepper_3d.py:367-393; DAMP: H' = d1 H - d2 curl
template <bool DAMP>
__global__ void __launch_bounds__(32 * SPLIT_Y, 2) k_yee3d_h(const __grid_constant__ Split3 P,
                                                             int i0) {
    const int nx = P.nx, ny = P.ny, nz = P.nz, ZP = P.zp;
    const int lane = threadIdx.x;
    const int j = blockIdx.y * SPLIT_Y + threadIdx.y;
    const int i = i0 + blockIdx.z;
    const int kb = blockIdx.x * 128 + 4 * lane;
    const bool act = j < ny && kb < ZP;
    const uint32_t NYZ = (uint32_t)ny * ZP;       // box < 2^31 elements (plan check)
    const uint32_t g = (uint32_t)i * NYZ + (uint32_t)(j * ZP + kb);
    const float dt = P.dt, rdx = P.rdx;
    const bool xok = i <= nx - 2, vyH = j <= ny - 2;
    const bool bx = xok && inband(P.B, 0, 0, i), by = vyH && inband(P.B, 1, 0, j);
    bool bz = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) bz |= kb + q <= nz - 2 && inband(P.B, 2, 0, kb + q);
    float ex[4], ey[4], ez[4], ezj[4], exj[4], ezi[4], eyi[4], hx[4], hy[4], hz[4];
    float p0[4], p1[4], p2[4], p3[4], p4[4], p5[4];
    float eyk = 0.f, exk = 0.f;
    z4(ex); z4(ey); z4(ez); z4(ezj); z4(exj); z4(ezi); z4(eyi); z4(hx); z4(hy); z4(hz);
    z4(p0); z4(p1); z4(p2); z4(p3); z4(p4); z4(p5);
    if (act) {
        ldg4v(P.e[0] + g, ex); ldg4v(P.e[1] + g, ey); ldg4v(P.e[2] + g, ez);
        if (j + 1 < ny) { ldg4v(P.e[2] + g + ZP, ezj); ldg4v(P.e[0] + g + ZP, exj); }
        if (i + 1 < nx) { ldg4v(P.e[2] + g + NYZ, ezi); ldg4v(P.e[1] + g + NYZ, eyi); }
        if (lane == 31 && kb + 4 < ZP) { eyk = __ldg(P.e[1] + g + 4); exk = __ldg(P.e[0] + g + 4); }
        ldg4v(P.h[0] + g, hx); ldg4v(P.h[1] + g, hy); ldg4v(P.h[2] + g, hz);
        if (by) ld4v(P.pi[0] + g, p0);
        if (vyH && bz) ld4v(P.pi[1] + g, p1);
        if (xok && bz) ld4v(P.pi[2] + g, p2);
        if (bx) ld4v(P.pi[3] + g, p3);
        if (vyH && bx) ld4v(P.pi[4] + g, p4);
        if (xok && by) ld4v(P.pi[5] + g, p5);
    }
    // profiles (tiny, cache resident); (1, 0) outside the bands
    float hxb = 1.f, hxa = 0.f, hyb = 1.f, hya = 0.f, hzb[4], hza[4];
    if (bx) { hxb = __ldg(P.pb[0][0] + i); hxa = __ldg(P.pa[0][0] + i); }
    if (by) { hyb = __ldg(P.pb[1][0] + j); hya = __ldg(P.pa[1][0] + j); }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const bool on = bz && kb + q <= nz - 2;
        hzb[q] = on ? __ldg(P.pb[2][0] + kb + q) : 1.f;
        hza[q] = on ? __ldg(P.pa[2][0] + kb + q) : 0.f;
    }
    {
        const float t0 = __shfl_down_sync(0xffffffffu, ey[0], 1);   // E(k+1) of q = 3
        const float t1 = __shfl_down_sync(0xffffffffu, ex[0], 1);
        if (lane != 31) { eyk = t0; exk = t1; }
    }
    if (!act) return;
    float a1[3][4], a2[3][4];
    if (DAMP) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            ldg4v(P.dmp[3 + c][0] + g, a1[c]);
            ldg4v(P.dmp[3 + c][1] + g, a2[c]);
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const bool vz = kb + q <= nz - 2, vzE = kb + q < nz;
        const float eyn = (q < 3) ? ey[q + 1] : eyk;
        const float exn = (q < 3) ? ex[q + 1] : exk;
        // Hx: valid j <= ny-2, k <= nz-2
        {
            float qy, qz;
            const float cu = __fsub_rn(y3_s(y3_d(ezj[q], ez[q], rdx), hyb, hya, p0[q], qy),
                                       y3_s(y3_d(eyn, ey[q], rdx), hzb[q], hza[q], p1[q], qz));
            const bool v = vyH && vz;
            const float hn = DAMP ? y3_hd(hx[q], cu, a1[0][q], a2[0][q]) : y3_h(hx[q], cu, dt);
            hx[q] = v ? hn : hx[q];
            p0[q] = v ? qy : p0[q];
            p1[q] = v ? qz : p1[q];
        }
        // Hy: valid i <= nx-2, k <= nz-2
        {
            float qz, qx;
            const float cu = __fsub_rn(y3_s(y3_d(exn, ex[q], rdx), hzb[q], hza[q], p2[q], qz),
                                       y3_s(y3_d(ezi[q], ez[q], rdx), hxb, hxa, p3[q], qx));
            const bool v = xok && vz;
            const float hn = DAMP ? y3_hd(hy[q], cu, a1[1][q], a2[1][q]) : y3_h(hy[q], cu, dt);
            hy[q] = v ? hn : hy[q];
            p2[q] = v ? qz : p2[q];
            p3[q] = v ? qx : p3[q];
        }
        // Hz: valid i <= nx-2, j <= ny-2, k < nz
        {
            float qx, qy;
            const float cu = __fsub_rn(y3_s(y3_d(eyi[q], ey[q], rdx), hxb, hxa, p4[q], qx),
                                       y3_s(y3_d(exj[q], ex[q], rdx), hyb, hya, p5[q], qy));
            const bool v = xok && vyH && vzE;
            const float hn = DAMP ? y3_hd(hz[q], cu, a1[2][q], a2[2][q]) : y3_h(hz[q], cu, dt);
            hz[q] = v ? hn : hz[q];
            p4[q] = v ? qx : p4[q];
            p5[q] = v ? qy : p5[q];
        }
    }
    st4v(P.ho[0] + g, hx);
    st4v(P.ho[1] + g, hy);
    st4v(P.ho[2] + g, hz);
    if (by) st4v(P.po[0] + g, p0);
    if (vyH && bz) st4v(P.po[1] + g, p1);
    if (xok && bz) st4v(P.po[2] + g, p2);
    if (bx) st4v(P.po[3] + g, p3);
    if (vyH && bx) st4v(P.po[4] + g, p4);
    if (xok && by) st4v(P.po[5] + g, p5);
}

// E(n+1) from H(n+1/2) and E(n): core/stepper_3d.py:395-437, source
// :448-482. The E-side psi recursions run over their arrays' full extent
// (core/stepper_3d.py:79-101 State3D shapes), wider than the interior where
// the curl is applied (_pad_interior). E(n+1) = E(n) + dt curl / eps_c with a
// fast (2 ulp) divide; the reference's (E eps + dt curl) / eps differs by
// rounding only.
template <int MODE>                 // bit 0: damping, bit 1: poles
__global__ void __launch_bounds__(32 * SPLIT_Y, 2) k_yee3d_e(const __grid_constant__ Split3 P,
                                                             const float *__restrict__ amp, int i0) {
    constexpr bool DAMP = (MODE & 1) != 0, PL = (MODE & 2) != 0;
    const int nx = P.nx, ny = P.ny, nz = P.nz, ZP = P.zp;
    const int lane = threadIdx.x;
    const int j = blockIdx.y * SPLIT_Y + threadIdx.y;
    const int i = i0 + blockIdx.z;
    const int kb = blockIdx.x * 128 + 4 * lane;
    const bool act = j < ny && kb < ZP;
    const uint32_t NYZ = (uint32_t)ny * ZP;       // box < 2^31 elements (plan check)
    const uint32_t g = (uint32_t)i * NYZ + (uint32_t)(j * ZP + kb);
    const float dt = P.dt, rdx = P.rdx;
    const bool iin = i >= 1 && i <= nx - 2, jin = j >= 1 && j <= ny - 2;
    const bool pmx = P.pmc & 1, pmy = (P.pmc >> 1) & 1, pmz = (P.pmc >> 2) & 1;
    const bool xok = i <= nx - 2, vyH = j <= ny - 2;
    const bool bx = iin && inband(P.B, 0, 1, i), by = jin && inband(P.B, 1, 1, j);
    bool bz = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = kb + q;
        bz |= k >= 1 && k <= nz - 2 && inband(P.B, 2, 1, k);
    }
    const float *__restrict__ Hx = P.ho[0];
    const float *__restrict__ Hy = P.ho[1];
    const float *__restrict__ Hz = P.ho[2];
    const float *__restrict__ eps = P.eps;
    float hx[4], hy[4], hz[4], ep[4], hzm[4], hxm[4], hzp[4], hyp[4], epj[4], epi[4], en[3][4];
    float p6[4], p7[4], p8[4], p9[4], p10[4], p11[4];
    float hyk = 0.f, hxk = 0.f, epk = 1.f;
    z4(hx); z4(hy); z4(hz); one4(ep); z4(hzm); z4(hxm); z4(hzp); z4(hyp); one4(epj); one4(epi);
    z4(p6); z4(p7); z4(p8); z4(p9); z4(p10); z4(p11);
    z4(en[0]); z4(en[1]); z4(en[2]);
    int e0 = 0, e1x = 0;                          // soft current cells of row (i, j)
    if (act) {
        ldg4v(Hx + g, hx); ldg4v(Hy + g, hy); ldg4v(Hz + g, hz); ldg4v(eps + g, ep);
        if (j >= 1) { ldg4v(Hz + g - ZP, hzm); ldg4v(Hx + g - ZP, hxm); }
        if (i >= 1) { ldg4v(Hz + g - NYZ, hzp); ldg4v(Hy + g - NYZ, hyp); }
        if (j + 1 < ny) ldg4v(eps + g + ZP, epj);
        if (i + 1 < nx) ldg4v(eps + g + NYZ, epi);
        if (lane == 0 && kb >= 1) { hyk = __ldg(Hy + g - 1); hxk = __ldg(Hx + g - 1); }
        if (lane == 31 && kb + 4 < ZP) epk = __ldg(eps + g + 4);
        ldg4v(P.e[0] + g, en[0]); ldg4v(P.e[1] + g, en[1]); ldg4v(P.e[2] + g, en[2]);
        if (xok && by) ld4v(P.pi[6] + g, p6);
        if (xok && bz) ld4v(P.pi[7] + g, p7);
        if (vyH && bz) ld4v(P.pi[8] + g, p8);
        if (vyH && bx) ld4v(P.pi[9] + g, p9);
        if (bx) ld4v(P.pi[10] + g, p10);
        if (by) ld4v(P.pi[11] + g, p11);
        if (P.src_n > 0) {
            e0 = __ldg(P.src_row + i * ny + j);
            e1x = __ldg(P.src_row + i * ny + j + 1);
        }
    }
    float exb = 1.f, exa = 0.f, eyb = 1.f, eya = 0.f, ezb[4], eza[4];
    if (bx) { exb = __ldg(P.pb[0][1] + i); exa = __ldg(P.pa[0][1] + i); }
    if (by) { eyb = __ldg(P.pb[1][1] + j); eya = __ldg(P.pa[1][1] + j); }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = kb + q;
        const bool on = bz && k >= 1 && k <= nz - 2;
        ezb[q] = on ? __ldg(P.pb[2][1] + k) : 1.f;
        eza[q] = on ? __ldg(P.pa[2][1] + k) : 0.f;
    }
    {
        const float t0 = __shfl_up_sync(0xffffffffu, hy[3], 1);     // H(k-1) of q = 0
        const float t1 = __shfl_up_sync(0xffffffffu, hx[3], 1);
        const float t2 = __shfl_down_sync(0xffffffffu, ep[0], 1);   // eps(k+1) of q = 3
        if (lane != 0) { hyk = t0; hxk = t1; }
        if (lane != 31) epk = t2;
    }
    if (!act) return;
    // conductive damping: E' = d1 E + d2 curl / eps (core/stepper_3d.py:405-437)
    float a1[3][4], a2[3][4];
    if (DAMP) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            ldg4v(P.dmp[c][0] + g, a1[c]);
            ldg4v(P.dmp[c][1] + g, a2[c]);
        }
    }
    // dispersive poles (core/stepper_3d.py:295-300, :312-325): P(n+1) = c1 P(n) +
    // c2 P(n-1) + c3 E(n) over the P(n-1) buffer, and the sums of P(n), P(n+1) that the
    // folded-D update E(n+1) = (d1 (eps E + sum P(n)) + d2 curl - sum P(n+1)) / eps needs
    float spc[3][4], spn[3][4];
    if (PL) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            z4(spc[c]);
            z4(spn[c]);
#pragma unroll 1
            for (int k = 0; k < P.np; ++k) {
                const uint32_t o = k * P.plane + g;
                float pc[4], pq[4], c3[4];
                ld4v(P.pp[c][0] + o, pc);
                ld4v(P.pp[c][1] + o, pq);
                ldg4v(P.pc3[c] + o, c3);
                const float c1 = P.pc1[k], c2 = P.pc2[k];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    spc[c][q] += pc[q];
                    pq[q] = __fmaf_rn(c3[q], en[c][q], __fmaf_rn(c2, pq[q], __fmul_rn(c1, pc[q])));
                    spn[c][q] += pq[q];
                }
                st4v(P.pp[c][1] + o, pq);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = kb + q;
        const bool vzE = k < nz, vz = k <= nz - 2, kin = k >= 1 && k <= nz - 2;
        const float hym = (q == 0) ? hyk : hy[q - 1];
        const float hxkm = (q == 0) ? hxk : hx[q - 1];
        // Ex: valid i <= nx-2, k < nz; curl on j, k interior
        {
            float qy, qz;
            const float ty = y3_s(y3_d(hz[q], hzm[q], rdx), eyb, eya, p6[q], qy);
            const float tz = y3_s(y3_d(hy[q], hym, rdx), ezb[q], eza[q], p7[q], qz);
            const bool v = xok && vzE;
            const float curl = y3_curl(ty, !jin, pmy, tz, !kin, pmz);
            const float ec = y3_ec(ep[q], epi[q]);
            en[0][q] = v ? (PL ? (DAMP ? y3_epd(en[0][q], curl, a1[0][q], a2[0][q], ec, spc[0][q],
                                                spn[0][q])
                                       : y3_ep(en[0][q], curl, dt, ec, spc[0][q], spn[0][q]))
                                 : DAMP ? y3_ed(en[0][q], curl, a1[0][q], a2[0][q], ec)
                                        : y3_e(en[0][q], curl, dt, ec))
                         : en[0][q];
            p6[q] = v ? qy : p6[q];
            p7[q] = v ? qz : p7[q];
        }
        // Ey: valid j <= ny-2, k < nz; curl on i, k interior
        {
            float qz, qx;
            const float tz = y3_s(y3_d(hx[q], hxkm, rdx), ezb[q], eza[q], p8[q], qz);
            const float tx = y3_s(y3_d(hz[q], hzp[q], rdx), exb, exa, p9[q], qx);
            const bool v = vyH && vzE;
            const float curl = y3_curl(tz, !kin, pmz, tx, !iin, pmx);
            const float ec = y3_ec(ep[q], epj[q]);
            en[1][q] = v ? (PL ? (DAMP ? y3_epd(en[1][q], curl, a1[1][q], a2[1][q], ec, spc[1][q],
                                                spn[1][q])
                                       : y3_ep(en[1][q], curl, dt, ec, spc[1][q], spn[1][q]))
                                 : DAMP ? y3_ed(en[1][q], curl, a1[1][q], a2[1][q], ec)
                                        : y3_e(en[1][q], curl, dt, ec))
                         : en[1][q];
            p8[q] = v ? qz : p8[q];
            p9[q] = v ? qx : p9[q];
        }
        // Ez: valid k <= nz-2; curl on i, j interior
        {
            float qx, qy;
            const float tx = y3_s(y3_d(hy[q], hyp[q], rdx), exb, exa, p10[q], qx);
            const float ty = y3_s(y3_d(hx[q], hxm[q], rdx), eyb, eya, p11[q], qy);
            const float curl = y3_curl(tx, !iin, pmx, ty, !jin, pmy);
            const float ec = y3_ec(ep[q], (q < 3) ? ep[q + 1] : epk);
            en[2][q] = vz ? (PL ? (DAMP ? y3_epd(en[2][q], curl, a1[2][q], a2[2][q], ec, spc[2][q],
                                                 spn[2][q])
                                        : y3_ep(en[2][q], curl, dt, ec, spc[2][q], spn[2][q]))
                                  : DAMP ? y3_ed(en[2][q], curl, a1[2][q], a2[2][q], ec)
                                         : y3_e(en[2][q], curl, dt, ec))
                          : en[2][q];
            p10[q] = vz ? qx : p10[q];
            p11[q] = vz ? qy : p11[q];
        }
    }
    // soft current cells of row (i, j) on component src_comp
    if (e0 < e1x) {
        const int c = P.src_comp;
        const float a = __ldg(amp);
        const float sgn = P.src_is_point ? (float)P.point_sign : -1.f;
        for (int e = e0; e < e1x; ++e) {
            const int kq = __ldg(P.src_col + e) - kb;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (kq != q) continue;
                float epn;
                if (c == 0) epn = epi[q];
                else if (c == 1) epn = epj[q];
                else epn = (q < 3) ? ep[q + 1] : epk;
                const float ecomp = y3_ec(ep[q], epn);
                const float v = __fmul_rn(a, __ldg(P.src_w + e));
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {         // static component index
                    if (cc != c) continue;
                    en[cc][q] = y3_src(en[cc][q], v, ecomp, P.src_is_point != 0, sgn);
                }
            }
        }
    }
    st4v(P.eo[0] + g, en[0]);
    st4v(P.eo[1] + g, en[1]);
    st4v(P.eo[2] + g, en[2]);
    if (xok && by) st4v(P.po[6] + g, p6);
    if (xok && bz) st4v(P.po[7] + g, p7);
    if (vyH && bz) st4v(P.po[8] + g, p8);
    if (vyH && bx) st4v(P.po[9] + g, p9);
    if (bx) st4v(P.po[10] + g, p10);
    if (by) st4v(P.po[11] + g, p11);
}

// Copy the plane samples of the (new) state into one ring slot.
__global__ void k_sample3d(const mtb_yee3d_struct *__restrict__ SS, const int64_t *__restrict__ pstart,
                           int n_planes, int cur, float *__restrict__ ring) {
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
    const float *F = S.f[comp][cur];
    ring[S.plane_ring_off[lo] + p] = F[((int64_t)i * S.ny + j) * S.zpitch + k];
}

}  // namespace mtb

#include "yee3d_xm.cuh"

using namespace mtb;

struct mtb_yee3d_plan {
    mtb_yee3d_struct s{};
    DevBuf s_d, pstart_d, amp_d;
    PinnedPair amp_h;
    int rows = 32;
    int nzw = 1;
    int variant = 2;               // 1 fused x-march, 2 split H / E, 3 one-pass TMA x-march
    bool chosen = false;           // variant 3 picked by default (half steps and slabs
                                   // fall back to the split kernels)
    XmMaps xm{};                   // variant 3: tensor maps of E (both buffers) and eps
    int xm_v = 0, xm_grid = 0, xm_tiles = 0;
    int xm_lock = 0;               // variant 3: x segments per tile of a lockstep geometry
    int xm_geom = 0;               // variant 3: asked geometry (mtb_tuning::geometry)
    DevBuf ytab_d;                 // variant 3: first row of each tile (XmMaps::ytab)
    DevBuf err_d;                  // variant 3: bounded-wait error flag
    DevBuf ptab_d;                 // variant 3: masked CPML profiles (XmMaps::ptab)
    DevBuf share_d;                // variant 3: unit range of each block (xm_grid + 1)
    Band3 band{};
    Split3 sp[2]{};                // split-kernel parameters of parity 0 and 1
    int slab = 0;                  // split kernels: x planes per H / E launch pair
    bool damp = false;             // conductive damping arrays given
    bool poles = false;            // dispersive pole stacks given
    int own_lo = 0, own_hi = 0;    // split kernels: x planes this plan updates
    // chunk staged by mtb_yee3d_begin: k steps from t0, next step c_s, next
    // half c_half (0 H, 1 E), ring slot c_slot
    int64_t c_t0 = 0;
    int c_k = 0, c_s = 0, c_half = 0, c_slot = 0;
    int par = 0;
    int n_planes = 0;
    int64_t n_samples = 0;
    size_t smem = 0;
    int64_t last_launches = 0;
    DftState dft;
    LaunchTimer timer;
};

// CPML band limits of one profile (device arrays of length len): every
// active node k (a != 0 or b != 1) satisfies k < lo or k >= hi.
static int profile_band3(const float *b_d, const float *a_d, int len, int &lo, int &hi) {
    std::vector<float> b(len), a(len);
    cudaError_t e = cudaMemcpy(b.data(), b_d, sizeof(float) * len, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(a.data(), a_d, sizeof(float) * len, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(MTB_CUDA_ERROR, "reading CPML profile: %s", cudaGetErrorString(e));
    lo = 0;
    hi = len;
    for (int k = 0; k < len / 2; ++k)
        if (a[k] != 0.f || b[k] != 1.f) lo = k + 1;
    for (int k = len - 1; k >= len / 2; --k)
        if (a[k] != 0.f || b[k] != 1.f) hi = k;
    return MTB_OK;
}

template <int NZW>
static int launch3d(mtb_yee3d_plan *p, Ctx3D C, cudaStream_t st) {
    const dim3 grid((p->s.ny + TY3 - 1) / TY3, (p->s.nx + p->rows - 1) / p->rows);
    k_yee3d_step<NZW><<<grid, 32 * NZW * (TY3 + 2), p->smem, st>>>(p->s_d.as<mtb_yee3d_struct>(),
                                                                    p->rows, C);
    MTB_CHECK_LAUNCH();
    return MTB_OK;
}

template <int NZW>
static int set_smem3d(size_t smem) {
    MTB_CUDA_TRY(cudaFuncSetAttribute(k_yee3d_step<NZW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    return MTB_OK;
}

// ---------------------------------------------------------------- one-pass x-march set-up
static PFN_cuTensorMapEncodeTiled_v12000 tmap3_encoder() {
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

// A 3D float32 tensor map over one box array (nx planes x ny rows x zp floats), box
// of bz x by x 1; reads outside the array return zero.
static int tmap_3d(CUtensorMap *m, const float *base, int nx, int ny, int zp, int bz, int by) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tmap3_encoder();
    if (!enc) return fail(MTB_CUDA_ERROR, "cuTensorMapEncodeTiled is not available");
    const cuuint64_t dims[3] = {(cuuint64_t)zp, (cuuint64_t)ny, (cuuint64_t)nx};
    const cuuint64_t strides[2] = {(cuuint64_t)zp * sizeof(float),
                                   (cuuint64_t)zp * ny * sizeof(float)};
    const cuuint32_t box[3] = {(cuuint32_t)bz, (cuuint32_t)by, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims,
                           strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(MTB_CUDA_ERROR, "3D tensor map encoding failed (%d)", (int)r);
    return MTB_OK;
}

// tile height per z width: (TY + 1) * V warps within 64 KB of registers without spills
template <int V> constexpr int xm_ty() { return V == 1 ? 8 : 5; }
static_assert(sizeof(Split3) + sizeof(XmMaps) + 64 <= 4096, "kernel parameters exceed 4 KB");

template <int V>
static int xm_setup(mtb_yee3d_plan *p) {
    constexpr int TY = xm_ty<V>();
    using Sh = XmShape<V, TY>;
    const mtb_yee3d_struct &S = p->s;
    int rc;
    // z-layer boxes: every float4 of z-layer cells (H or E side) lies below zl or at /
    // above zh, both multiples of 4, each box XM_BZ wide
    const Band3 &B = p->band;
    const int lo = std::max(B.lo[2][0], B.lo[2][1]), hi = std::min(B.hi[2][0], B.hi[2][1]);
    const int zl = (lo + 3) / 4 * 4, zh = hi / 4 * 4;
    p->xm.npz = (lo > 0 || hi < S.nz - 1) ? 1 : 0;
    p->xm.zl = p->xm.npz ? zl : 0;
    p->xm.zh = p->xm.npz ? zh : (1 << 30);
    if (p->xm.npz && (zl > XM_BZ || S.zpitch - zh > XM_BZ || zh < 0))
        return fail(MTB_UNSUPPORTED, "one-pass 3D kernel: z CPML layers wider than %d cells",
                    XM_BZ - 4);
    for (int b = 0; b < 2; ++b) {
        for (int c = 0; c < 3; ++c) {
            if ((rc = tmap_3d(&p->xm.e[b][c], S.f[c][b], S.nx, S.ny, S.zpitch, Sh::ZB, Sh::EROWS)) ||
                (rc = tmap_3d(&p->xm.h[b][c], S.f[3 + c][b], S.nx, S.ny, S.zpitch, Sh::ZB,
                              Sh::SLOTS)))
                return rc;
        }
        const int pzi[4] = {1, 2, 7, 8};
        for (int a = 0; a < 4; ++a)
            if ((rc = tmap_3d(&p->xm.pz[b][a], S.psi[pzi[a]][b], S.nx, S.ny, S.zpitch, XM_BZ,
                              Sh::SLOTS)))
                return rc;
    }
    if ((rc = tmap_3d(&p->xm.eps, S.eps, S.nx, S.ny, S.zpitch, Sh::ZB, Sh::PROWS))) return rc;
    // profiles as the split kernels apply them: the H-side node k of an axis of n cells
    // is updated for k <= n-2, the E-side curl for 1 <= k <= n-2; (1, 0) elsewhere
    {
        const int dims[3] = {S.nx, S.ny, S.zpitch};
        const int real[3] = {S.nx, S.ny, S.nz};
        std::vector<float> tab;
        for (int a = 0; a < 3; ++a) {
            const int n = dims[a], nr = real[a];
            std::vector<float> prof[2][2];
            for (int h = 0; h < 2; ++h) {
                const int len = nr - 1 + h;
                for (int v = 0; v < 2; ++v) {
                    prof[h][v].resize(len);
                    const float *src = v ? S.prof_a[a][h] : S.prof_b[a][h];
                    MTB_CUDA_TRY(cudaMemcpy(prof[h][v].data(), src, sizeof(float) * len,
                                            cudaMemcpyDeviceToHost));
                }
            }
            for (int h = 0; h < 2; ++h)
                for (int v = 0; v < 2; ++v)
                    for (int k = 0; k < n; ++k) {
                        const bool on = h == 0 ? k <= nr - 2 : (k >= 1 && k <= nr - 2);
                        tab.push_back(on ? prof[h][v][k] : (v ? 0.f : 1.f));
                    }
        }
        if ((rc = p->ptab_d.ensure(sizeof(float) * tab.size()))) return rc;
        MTB_CUDA_TRY(cudaMemcpy(p->ptab_d.p, tab.data(), sizeof(float) * tab.size(),
                                cudaMemcpyHostToDevice));
        p->xm.ptab = p->ptab_d.as<float>();
    }
    MTB_CUDA_TRY(cudaFuncSetAttribute(k_yee3d_xm<V, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)Sh::SMEM));
    int dev = 0, sms = 0, occ = 0;
    MTB_CUDA_TRY(cudaGetDevice(&dev));
    MTB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MTB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_yee3d_xm<V, TY>, Sh::THREADS,
                                                               Sh::SMEM));
    if (occ < 1) return fail(MTB_UNSUPPORTED, "one-pass 3D kernel does not fit on an SM");
    // Work geometry. A (tile, plane) pair costs XM_LAYER_COST per row in an x / y CPML
    // layer (memory read from HBM, the full update), 1 per other row, the recomputed
    // halo row included.
    //  - lockstep: G x segments (the same cuts for every tile, equal x cost) times T
    //    tiles of at most TY rows whose costs are balanced, G * T <= the resident
    //    blocks; y-neighbour tiles then pass each plane together and the halo rows
    //    one reads come from L2 (written or read by the other a moment before);
    //  - otherwise TY-row tiles and one tile-major share of equal cost per resident
    //    block (at least four planes each).
    // The default is tile-major: measured on the 256^3 and 192^3 grids, lockstep cuts
    // the DRAM bytes from 1.18-1.22x to 1.03x of the algorithmic bytes but runs
    // 1.3-1.4x longer (its 2-4 row tiles leave warps idle and the kernel is bound by
    // instruction issue, not DRAM), so it is only taken when asked for.
    constexpr double XM_LAYER_COST = 1.6;
    auto band = [&](int a, int k) {
        return k < B.lo[a][0] || k >= B.hi[a][0] || k < B.lo[a][1] || k >= B.hi[a][1];
    };
    const int cap = sms * occ;
    std::vector<double> cy(S.ny), cxp(S.nx + 1, 0.0);
    for (int r = 0; r < S.ny; ++r) cy[r] = band(1, r) ? XM_LAYER_COST : 1.0;
    for (int i = 0; i < S.nx; ++i) cxp[i + 1] = cxp[i] + (band(0, i) ? XM_LAYER_COST : 1.0);
    // tile-major reference: TY-row tiles, equal-cost shares
    const int t_uni = (S.ny + TY - 1) / TY;
    double rows_uni = 0.0;
    for (int r = 0; r < S.ny; ++r) rows_uni += cy[r];
    rows_uni += (t_uni - 1) * 1.0;                         // recomputed halo rows
    const double cost_uni = rows_uni * cxp[S.nx] / std::max(1, cap);
    // lockstep candidates: min-max partition of the rows into T tiles of <= TY rows
    auto partition = [&](int T, std::vector<int> &y0s) -> double {
        auto tile_cost = [&](int a, int b) {          // rows a .. b-1 plus halo a-1
            double c = a > 0 ? cy[a - 1] : 0.0;
            for (int r = a; r < b; ++r) c += cy[r];
            return c;
        };
        auto fits = [&](double lim, std::vector<int> *out) {
            int a = 0, n = 0;
            if (out) out->assign(1, 0);
            while (a < S.ny) {
                int b = a + 1;
                if (tile_cost(a, b) > lim) return false;
                while (b < S.ny && b - a < TY && tile_cost(a, b + 1) <= lim) ++b;
                a = b;
                ++n;
                if (out) out->push_back(a);
            }
            return n <= T;
        };
        double lo = 0.0, hi = (TY + 1) * XM_LAYER_COST;
        if (!fits(hi, nullptr)) return -1.0;
        for (int it = 0; it < 40; ++it) {
            const double mid = 0.5 * (lo + hi);
            if (fits(mid, nullptr)) hi = mid; else lo = mid;
        }
        fits(hi, &y0s);
        return hi;
    };
    int best_g = 0;
    double best_cost = 0.0;
    std::vector<int> best_y0;
    for (int G = 1; G <= 8; ++G) {
        const int T = cap / G;
        if (T < 1 || (int64_t)T * TY < S.ny || S.nx / G < 4) continue;
        std::vector<int> y0s;
        const double tc = partition(T, y0s);
        if (tc < 0) continue;
        const double c = tc * cxp[S.nx] / G;
        if (!best_g || c < best_cost) { best_g = G; best_cost = c; best_y0 = y0s; }
    }
    std::vector<int> ytab;
    std::vector<int64_t> share;
    p->xm_v = V;
    if (p->xm_geom < 0 || p->xm_geom > 2)
        return fail(MTB_INVALID_ARG, "3D geometry %d not in 0..2", p->xm_geom);
    if (p->xm_geom == 2 && !best_g)
        return fail(MTB_UNSUPPORTED, "no lockstep geometry for this grid");
    (void)cost_uni;
    if (best_g && p->xm_geom == 2) {
        const int G = best_g;
        ytab = best_y0;
        p->xm_tiles = (int)ytab.size() - 1;
        std::vector<int> cut(G + 1);
        for (int g = 0, i = 0; g <= G; ++g) {
            const double target = cxp[S.nx] * g / G;
            while (i < S.nx && cxp[i] < target) ++i;
            cut[g] = (g == G) ? S.nx : i;
        }
        for (int t = 0; t < p->xm_tiles; ++t)
            for (int g = 0; g < G; ++g)
                if (cut[g + 1] > cut[g]) share.push_back((int64_t)t * S.nx + cut[g]);
        share.push_back((int64_t)p->xm_tiles * S.nx);
        p->xm_lock = G;
    } else {
        p->xm_tiles = t_uni;
        for (int t = 0; t <= t_uni; ++t) ytab.push_back(std::min(t * TY, S.ny));
        const int64_t units = (int64_t)t_uni * S.nx;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(cap, units / 4));
        std::vector<double> cum(units + 1, 0.0);
        for (int64_t u = 0; u < units; ++u) {
            const int t = (int)(u / S.nx), i = (int)(u % S.nx);
            bool yb = false;
            for (int r = std::max(ytab[t] - 1, 0); r < ytab[t + 1]; ++r) yb |= band(1, r);
            cum[u + 1] = cum[u] + ((band(0, i) || yb) ? XM_LAYER_COST : 1.0);
        }
        int64_t u = 0;
        for (int b = 0; b <= grid; ++b) {
            const double target = cum[units] * b / grid;
            while (u < units && cum[u] < target) ++u;
            share.push_back(b == grid ? units : u);
        }
        p->xm_lock = 0;
    }
    p->xm_grid = (int)share.size() - 1;
    if ((rc = p->share_d.ensure(sizeof(int64_t) * share.size()))) return rc;
    MTB_CUDA_TRY(cudaMemcpy(p->share_d.p, share.data(), sizeof(int64_t) * share.size(),
                            cudaMemcpyHostToDevice));
    if ((rc = p->ytab_d.ensure(sizeof(int) * ytab.size()))) return rc;
    MTB_CUDA_TRY(cudaMemcpy(p->ytab_d.p, ytab.data(), sizeof(int) * ytab.size(),
                            cudaMemcpyHostToDevice));
    p->xm.ytab = p->ytab_d.as<int>();
    return p->err_d.ensure(sizeof(int));
}

static int launch_xm(mtb_yee3d_plan *p, int s, cudaStream_t st) {
    const float *a = p->amp_d.as<float>() + s;
    using S1 = XmShape<1, xm_ty<1>()>;
    using S2 = XmShape<2, xm_ty<2>()>;
    if (p->xm_v == 1)
        k_yee3d_xm<1, xm_ty<1>()><<<p->xm_grid, S1::THREADS, S1::SMEM, st>>>(
            p->sp[p->par], p->xm, a, p->par, p->share_d.as<int64_t>(), p->err_d.as<int>());
    else
        k_yee3d_xm<2, xm_ty<2>()><<<p->xm_grid, S2::THREADS, S2::SMEM, st>>>(
            p->sp[p->par], p->xm, a, p->par, p->share_d.as<int64_t>(), p->err_d.as<int>());
    MTB_CHECK_LAUNCH();
    ++p->last_launches;
    return MTB_OK;
}

extern "C" {

int mtb_yee3d_plan_create(const mtb_yee3d_struct *s, const mtb_dft_region *regions,
                          int32_t n_regions, const mtb_phase_group *groups, int32_t n_groups,
                          int64_t ring_slot_elems, const mtb_tuning *tuning,
                          mtb_yee3d_plan **out) {
    if (!out || !s) return fail(MTB_INVALID_ARG, "null argument");
    *out = nullptr;
    const mtb_yee3d_struct &S = *s;
    if (S.nx < 3 || S.ny < 3 || S.nz < 3)
        return fail(MTB_INVALID_ARG, "nx, ny, nz must be >= 3");
    if (S.zpitch < S.nz || (S.zpitch & 3))
        return fail(MTB_INVALID_ARG, "zpitch %d must be >= nz and a multiple of 4", S.zpitch);
    // variant 3 (one pass per step) by default where it applies: no conductive
    // damping or poles, zpitch <= 256
    const int asked = tuning ? tuning->variant : 0;
    if (asked < 0 || asked > 3) return fail(MTB_INVALID_ARG, "3D variant %d not in 0..3", asked);
    int n_damp0 = 0;
    for (int c = 0; c < 6; ++c)
        for (int h = 0; h < 2; ++h) n_damp0 += S.damp[c][h] != nullptr;
    const bool xm_ok = n_damp0 == 0 && S.n_poles == 0 && S.zpitch <= 256;
    if (asked == 3 && !xm_ok)
        return fail(MTB_UNSUPPORTED, "one-pass 3D kernel: no damping or poles, zpitch <= 256");
    const int variant = asked == 1 ? 1 : (asked == 3 || (asked == 0 && xm_ok)) ? 3 : 2;
    if (variant == 1 && S.zpitch > 128 * MAXNZ)
        return fail(MTB_UNSUPPORTED, "fused kernel: zpitch %d > %d not supported", S.zpitch,
                    128 * MAXNZ);
    if (variant != 1 && (S.nx > 65535 || (S.ny + SPLIT_Y - 1) / SPLIT_Y > 65535 ||
                         (int64_t)S.nx * S.ny * S.zpitch >= (1LL << 31)))
        return fail(MTB_UNSUPPORTED, "split kernels: nx <= 65535, ny <= %d, box < 2^31 cells",
                    65535 * SPLIT_Y);
    if ((int64_t)S.nx * S.ny * S.zpitch >= (1LL << 34))
        return fail(MTB_UNSUPPORTED, "grid too large");
    if ((int64_t)S.nx * S.ny >= (1LL << 31)) return fail(MTB_UNSUPPORTED, "nx*ny too large");
    if (!(S.dt > 0.f) || !(S.dx > 0.f)) return fail(MTB_INVALID_ARG, "dt, dx must be > 0");
    if (S.point_sign != 1 && S.point_sign != -1)
        return fail(MTB_INVALID_ARG, "point_sign must be +1 or -1");
    for (int c = 0; c < 6; ++c)
        for (int b = 0; b < 2; ++b)
            if (!S.f[c][b] || (reinterpret_cast<uintptr_t>(S.f[c][b]) & 15))
                return fail(MTB_INVALID_ARG, "field %d buffer %d null or not 16-byte aligned", c, b);
    for (int c = 0; c < 12; ++c)
        for (int b = 0; b < 2; ++b)
            if (!S.psi[c][b] || (reinterpret_cast<uintptr_t>(S.psi[c][b]) & 15))
                return fail(MTB_INVALID_ARG, "psi %d buffer %d null or not 16-byte aligned", c, b);
    if (!S.eps || (reinterpret_cast<uintptr_t>(S.eps) & 15))
        return fail(MTB_INVALID_ARG, "eps null or not 16-byte aligned");
    for (int a = 0; a < 3; ++a)
        for (int h = 0; h < 2; ++h)
            if (!S.prof_b[a][h] || !S.prof_a[a][h])
                return fail(MTB_INVALID_ARG, "null CPML profile");
    if (S.src.n < 0) return fail(MTB_INVALID_ARG, "negative source cell count");
    if (S.src.n > 0) {
        if (!S.src.row_ptr || !S.src.col || !S.src.w || S.src.amp_col != 0)
            return fail(MTB_INVALID_ARG, "source cells: null arrays or amp_col != 0");
        if (S.src_comp < 0 || S.src_comp > 2)
            return fail(MTB_INVALID_ARG, "src_comp must be Ex, Ey or Ez");
    }
    if (S.n_planes < 0 || (S.n_planes > 0 && (!S.planes || !S.plane_ring_off)))
        return fail(MTB_INVALID_ARG, "bad plane sample list");
    int n_damp = 0;
    for (int c = 0; c < 6; ++c)
        for (int h = 0; h < 2; ++h) {
            if (!S.damp[c][h]) continue;
            ++n_damp;
            if (reinterpret_cast<uintptr_t>(S.damp[c][h]) & 15)
                return fail(MTB_INVALID_ARG, "damping array %d/%d not 16-byte aligned", c, h);
        }
    if (n_damp != 0 && n_damp != 12)
        return fail(MTB_INVALID_ARG, "damping: give all 12 (d1, d2) arrays or none");
    if (n_damp && variant == 1)
        return fail(MTB_UNSUPPORTED, "conductive damping needs the split kernels");
    if (S.pmc_axes < 0 || S.pmc_axes > 7)
        return fail(MTB_INVALID_ARG, "pmc_axes %d is not a mask of x / y / z", S.pmc_axes);
    if (S.pmc_axes && variant == 1)
        return fail(MTB_UNSUPPORTED, "PMC walls need the split or one-pass kernels");
    if (S.n_poles < 0 || S.n_poles > MTB_MAX_POLES)
        return fail(MTB_INVALID_ARG, "n_poles %d outside [0, %d]", S.n_poles, MTB_MAX_POLES);
    if (S.n_poles > 0) {
        if (variant == 1) return fail(MTB_UNSUPPORTED, "poles need the split kernels");
        for (int c = 0; c < 3; ++c) {
            for (int b = 0; b < 2; ++b)
                if (!S.pol_p[c][b] || (reinterpret_cast<uintptr_t>(S.pol_p[c][b]) & 15))
                    return fail(MTB_INVALID_ARG, "pole buffer %d/%d null or misaligned", c, b);
            if (!S.pol_c3[c] || (reinterpret_cast<uintptr_t>(S.pol_c3[c]) & 15))
                return fail(MTB_INVALID_ARG, "pole c3 %d null or misaligned", c);
        }
        if ((int64_t)S.n_poles * S.nx * S.ny * S.zpitch >= (1LL << 31))
            return fail(MTB_UNSUPPORTED, "pole stacks too large");
    }
    mtb_yee3d_plan *p = new mtb_yee3d_plan();
    p->s = S;
    p->rows = (tuning && tuning->rows_per_warp > 0) ? tuning->rows_per_warp : 32;
    p->variant = variant;
    p->chosen = variant == 3 && asked == 0;
    p->xm_geom = tuning ? tuning->geometry : 0;
    // split kernels: rows_per_warp > 0 sets the x planes per launch pair; the
    // default is the whole grid in one pair
    p->slab = (tuning && tuning->rows_per_warp > 0) ? std::min(tuning->rows_per_warp, S.nx) : S.nx;
    p->own_lo = 0;
    p->own_hi = S.nx;
    p->damp = n_damp == 12;
    p->poles = S.n_poles > 0;
    const int slots = (tuning && tuning->ring_slots > 0) ? tuning->ring_slots : 32;
    p->nzw = (S.zpitch + 127) / 128;
    p->smem = sizeof(float) * (size_t)(S.zpitch + 4) * (4 * (TY3 + 2) + 3 * (TY3 + 1));
    p->n_planes = S.n_planes;
    int rc = p->dft.init(regions, n_regions, groups, n_groups, ring_slot_elems, slots);
    if (!rc) rc = p->s_d.ensure(sizeof(mtb_yee3d_struct));
    if (!rc) rc = p->pstart_d.ensure(sizeof(int64_t) * (S.n_planes + 1));
    if (!rc && variant != 1) {
        const int dims[3] = {S.nx, S.ny, S.nz};
        for (int a = 0; a < 3 && !rc; ++a)
            for (int h = 0; h < 2 && !rc; ++h)
                rc = profile_band3(S.prof_b[a][h], S.prof_a[a][h], dims[a] - 1 + h,
                                   p->band.lo[a][h], p->band.hi[a][h]);
    }
    if (!rc && variant != 1) {
        for (int par = 0; par < 2; ++par) {
            Split3 &q = p->sp[par];
            for (int c = 0; c < 3; ++c) {
                q.e[c] = S.f[c][par];
                q.eo[c] = S.f[c][par ^ 1];
                q.h[c] = S.f[3 + c][par];
                q.ho[c] = S.f[3 + c][par ^ 1];
            }
            for (int c = 0; c < 12; ++c) {
                q.pi[c] = S.psi[c][par];
                q.po[c] = S.psi[c][par ^ 1];
            }
            q.eps = S.eps;
            for (int a = 0; a < 3; ++a)
                for (int h = 0; h < 2; ++h) {
                    q.pb[a][h] = S.prof_b[a][h];
                    q.pa[a][h] = S.prof_a[a][h];
                }
            q.src_row = S.src.row_ptr;
            q.src_col = S.src.col;
            q.src_w = S.src.w;
            q.src_n = S.src.n;
            q.src_comp = S.src_comp;
            q.src_is_point = S.src_is_point;
            q.point_sign = S.point_sign;
            q.nx = S.nx; q.ny = S.ny; q.nz = S.nz; q.zp = S.zpitch;
            q.dt = S.dt;
            q.rdx = 1.0f / S.dx;
            q.B = p->band;
            for (int c = 0; c < 6; ++c)
                for (int h = 0; h < 2; ++h) q.dmp[c][h] = S.damp[c][h];
            q.np = S.n_poles;
            q.plane = (uint32_t)((int64_t)S.nx * S.ny * S.zpitch);
            q.pmc = S.pmc_axes;
            for (int c = 0; c < 3; ++c) {
                q.pp[c][0] = S.pol_p[c][par];
                q.pp[c][1] = S.pol_p[c][par ^ 1];
                q.pc3[c] = S.pol_c3[c];
            }
            for (int k = 0; k < MTB_MAX_POLES; ++k) {
                q.pc1[k] = k < S.n_poles ? S.pol_c1[k] : 0.f;
                q.pc2[k] = k < S.n_poles ? S.pol_c2[k] : 0.f;
            }
        }
    }
    if (!rc && variant == 1) {
        switch (p->nzw) {
            case 1: rc = set_smem3d<1>(p->smem); break;
            case 2: rc = set_smem3d<2>(p->smem); break;
            case 3: rc = set_smem3d<3>(p->smem); break;
            default: rc = set_smem3d<4>(p->smem); break;
        }
    }
    if (!rc && variant == 3) {
        rc = S.zpitch <= 128 ? xm_setup<1>(p) : xm_setup<2>(p);
        if (rc && p->chosen) {          // default choice only: keep the split kernels
            rc = MTB_OK;
            p->variant = 2;
            p->chosen = false;
        }
    }
    if (rc) { mtb_yee3d_plan_destroy(p); return rc; }
    // plane sample extents (host copy of the device list)
    std::vector<int64_t> ps(S.n_planes + 1, 0);
    if (S.n_planes > 0) {
        std::vector<int32_t> pl(8 * S.n_planes);
        cudaError_t e = cudaMemcpy(pl.data(), S.planes, sizeof(int32_t) * 8 * S.n_planes,
                                   cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            mtb_yee3d_plan_destroy(p);
            return fail(MTB_CUDA_ERROR, "reading plane list: %s", cudaGetErrorString(e));
        }
        const int dims[3] = {S.nx, S.ny, S.nz};
        for (int q = 0; q < S.n_planes; ++q) {
            const int *d = &pl[8 * q];
            const int comp = d[0], axis = d[1], index = d[2];
            const int a0 = (axis == 0) ? 1 : 0, a1 = (axis == 2) ? 1 : 2;
            if (comp < 0 || comp > 5 || axis < 0 || axis > 2 || index < 0 ||
                index >= dims[axis] || d[3] < 0 || d[4] > dims[a0] || d[3] > d[4] || d[5] < 0 ||
                d[6] > dims[a1] || d[5] > d[6]) {
                mtb_yee3d_plan_destroy(p);
                return fail(MTB_INVALID_ARG, "plane sample %d out of range", q);
            }
            ps[q + 1] = ps[q] + (int64_t)(d[4] - d[3]) * (d[6] - d[5]);
        }
    }
    p->n_samples = ps[S.n_planes];
    cudaError_t e = cudaMemcpy(p->s_d.p, &S, sizeof(S), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(p->pstart_d.p, ps.data(), sizeof(int64_t) * ps.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && p->err_d.p) e = cudaMemset(p->err_d.p, 0, sizeof(int));
    if (e != cudaSuccess) {
        mtb_yee3d_plan_destroy(p);
        return fail(MTB_CUDA_ERROR, "plan upload failed: %s", cudaGetErrorString(e));
    }
    *out = p;
    return MTB_OK;
}

}  // extern "C"

// Stage the source amplitudes and DFT phases of steps [t0, t0+k) on `st`.
static int stage_chunk(mtb_yee3d_plan *p, int64_t t0, int k, const double *coef, cudaStream_t st) {
    int rc;
    void *hp = nullptr;
    if ((rc = p->amp_h.acquire(sizeof(float) * k, &hp))) return rc;
    if ((rc = p->amp_d.ensure(sizeof(float) * k))) return rc;
    if ((rc = p->dft.upload_phases(t0, k, st))) return rc;
    float *ah = static_cast<float *>(hp);
    for (int s = 0; s < k; ++s) ah[s] = coef ? (float)coef[s] : 0.f;
    MTB_CUDA_TRY(cudaMemcpyAsync(p->amp_d.p, ah, sizeof(float) * k, cudaMemcpyHostToDevice, st));
    if ((rc = p->amp_h.queued(st))) return rc;
    p->c_t0 = t0;
    p->c_k = k;
    p->c_s = 0;
    p->c_half = 0;
    p->c_slot = 0;
    return MTB_OK;
}

// Split-kernel H (part 0) or E (part 1) update of x planes [i0, i1), step s
// of the staged chunk.
static int launch_split(mtb_yee3d_plan *p, int part, int i0, int i1, int s, cudaStream_t st) {
    if (i1 <= i0) return MTB_OK;
    const dim3 grid((p->s.zpitch + 127) / 128, (p->s.ny + SPLIT_Y - 1) / SPLIT_Y, i1 - i0);
    const dim3 block(32, SPLIT_Y);
    if (part == 0) {
        if (p->damp)
            k_yee3d_h<true><<<grid, block, 0, st>>>(p->sp[p->par], i0);
        else
            k_yee3d_h<false><<<grid, block, 0, st>>>(p->sp[p->par], i0);
    } else {
        const float *a = p->amp_d.as<float>() + s;
        switch ((p->damp ? 1 : 0) | (p->poles ? 2 : 0)) {
            case 0: k_yee3d_e<0><<<grid, block, 0, st>>>(p->sp[p->par], a, i0); break;
            case 1: k_yee3d_e<1><<<grid, block, 0, st>>>(p->sp[p->par], a, i0); break;
            case 2: k_yee3d_e<2><<<grid, block, 0, st>>>(p->sp[p->par], a, i0); break;
            default: k_yee3d_e<3><<<grid, block, 0, st>>>(p->sp[p->par], a, i0); break;
        }
    }
    MTB_CHECK_LAUNCH();
    ++p->last_launches;
    return MTB_OK;
}

// After the E update of step c_s: flip the buffers, sample the planes into
// the ring, fold a full ring (or the chunk's last steps) into the accumulators.
static int finish_step(mtb_yee3d_plan *p, cudaStream_t st) {
    int rc;
    p->par ^= 1;
    const bool sampling = p->dft.n_regions > 0 && p->n_samples > 0;
    if (sampling) {
        float *ring = p->dft.ring_d.as<float>() + (size_t)p->c_slot * p->dft.slot_elems;
        const int64_t nb = (p->n_samples + 255) / 256;
        k_sample3d<<<(unsigned)nb, 256, 0, st>>>(p->s_d.as<mtb_yee3d_struct>(),
                                                p->pstart_d.as<int64_t>(), p->n_planes, p->par,
                                                ring);
        MTB_CHECK_LAUNCH();
        ++p->last_launches;
    }
    const int s = p->c_s;
    ++p->c_slot;
    if (p->c_slot == p->dft.slots || s == p->c_k - 1) {
        if (sampling) {
            if ((rc = p->dft.contract(s + 1 - p->c_slot, p->c_slot, st, &p->timer))) return rc;
            ++p->last_launches;
        }
        p->c_slot = 0;
    }
    ++p->c_s;
    p->c_half = 0;
    return p->c_s == p->c_k ? p->timer.collect() : MTB_OK;
}

extern "C" {

int mtb_yee3d_run(mtb_yee3d_plan *p, int64_t t0, int32_t k, const double *coef, void *stream) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    if (k < 0) return fail(MTB_INVALID_ARG, "k < 0");
    p->last_launches = 0;
    if (k == 0) return MTB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    if ((rc = stage_chunk(p, t0, k, coef, st))) return rc;
    for (int s = 0; s < k; ++s) {
        if ((rc = p->timer.begin(st, 0))) return rc;
        if (p->variant == 3) {
            if ((rc = launch_xm(p, s, st))) return rc;
        } else if (p->variant == 1) {
            Ctx3D C;
            C.amp = p->amp_d.as<float>() + s;
            C.par = p->par;
            switch (p->nzw) {
                case 1: rc = launch3d<1>(p, C, st); break;
                case 2: rc = launch3d<2>(p, C, st); break;
                case 3: rc = launch3d<3>(p, C, st); break;
                default: rc = launch3d<4>(p, C, st); break;
            }
            if (rc) return rc;
            ++p->last_launches;
        } else {
            // x slabs: H(slab) then E(slab), so the E kernel finds E(n) and
            // H(n+1/2) of its planes in L2. E(slab) needs H of the slab and of
            // the plane before it, which the previous slab wrote.
            const int ns = p->slab;
            for (int i0 = p->own_lo; i0 < p->own_hi; i0 += ns) {
                const int i1 = std::min(i0 + ns, p->own_hi);
                if ((rc = launch_split(p, 0, i0, i1, s, st))) return rc;
                if ((rc = launch_split(p, 1, i0, i1, s, st))) return rc;
            }
        }
        if ((rc = p->timer.end(st))) return rc;
        if ((rc = finish_step(p, st))) return rc;
    }
    return MTB_OK;
}

int mtb_yee3d_check(mtb_yee3d_plan *p, void *stream) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    if (!p->err_d.p) return MTB_OK;
    int flag = 0;
    MTB_CUDA_TRY(cudaMemcpyAsync(&flag, p->err_d.p, sizeof(int), cudaMemcpyDeviceToHost,
                                 (cudaStream_t)stream));
    MTB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    if (flag)
        return fail(MTB_DEVICE_TIMEOUT, "a bounded wait for a staged plane copy expired on the "
                    "device; the affected steps are incomplete");
    return MTB_OK;
}

// Half steps and x slabs run on the split kernels: a plan that took the one-pass
// kernel by default moves to them (same results); an explicit request is refused.
static int need_split(mtb_yee3d_plan *p, const char *what) {
    if (p->variant == 3 && p->chosen) p->variant = 2;
    if (p->variant != 2) return fail(MTB_UNSUPPORTED, "%s need the split kernels", what);
    return MTB_OK;
}

int mtb_yee3d_set_slab(mtb_yee3d_plan *p, int32_t own_lo, int32_t own_hi) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    if (int rc = need_split(p, "x slabs")) return rc;
    if (own_lo < 0 || own_hi > p->s.nx || own_lo >= own_hi)
        return fail(MTB_INVALID_ARG, "slab [%d, %d) outside [0, %d)", own_lo, own_hi, p->s.nx);
    p->own_lo = own_lo;
    p->own_hi = own_hi;
    return MTB_OK;
}

int mtb_yee3d_begin(mtb_yee3d_plan *p, int64_t t0, int32_t k, const double *coef, void *stream) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    if (int rc = need_split(p, "half steps")) return rc;
    if (k <= 0) return fail(MTB_INVALID_ARG, "k must be > 0");
    p->last_launches = 0;
    return stage_chunk(p, t0, k, coef, (cudaStream_t)stream);
}

int mtb_yee3d_half(mtb_yee3d_plan *p, int32_t part, void *stream) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    if (p->c_s >= p->c_k) return fail(MTB_INVALID_ARG, "no staged step left (mtb_yee3d_begin)");
    if (part != p->c_half)
        return fail(MTB_INVALID_ARG, "half %d out of order (expected %d)", part, p->c_half);
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    if (part == 0) {
        if ((rc = p->timer.begin(st, 0))) return rc;
        if ((rc = launch_split(p, 0, p->own_lo, p->own_hi, p->c_s, st))) return rc;
        p->c_half = 1;
        return MTB_OK;
    }
    if ((rc = launch_split(p, 1, p->own_lo, p->own_hi, p->c_s, st))) return rc;
    if ((rc = p->timer.end(st))) return rc;
    return finish_step(p, st);
}

int mtb_yee3d_set_timing(mtb_yee3d_plan *p, int32_t enable) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    p->timer.on = enable != 0;
    p->timer.ms[0] = p->timer.ms[1] = 0;
    p->timer.count[0] = p->timer.count[1] = 0;
    return MTB_OK;
}

int mtb_yee3d_timing(const mtb_yee3d_plan *p, double *step_ms, int64_t *step_launches,
                     double *dft_ms, int64_t *dft_launches) {
    if (!p) return fail(MTB_INVALID_ARG, "plan is null");
    if (step_ms) *step_ms = p->timer.ms[0];
    if (step_launches) *step_launches = p->timer.count[0];
    if (dft_ms) *dft_ms = p->timer.ms[1];
    if (dft_launches) *dft_launches = p->timer.count[1];
    return MTB_OK;
}

int32_t mtb_yee3d_current(const mtb_yee3d_plan *p) { return p ? p->par : -1; }

int64_t mtb_yee3d_last_launches(const mtb_yee3d_plan *p) { return p ? p->last_launches : -1; }

void mtb_yee3d_plan_destroy(mtb_yee3d_plan *p) {
    if (!p) return;
    p->s_d.release();
    p->pstart_d.release();
    p->amp_d.release();
    p->amp_h.release();
    p->dft.release();
    p->timer.release();
    p->err_d.release();
    p->ptab_d.release();
    p->share_d.release();
    p->ytab_d.release();
    delete p;
}

}  // extern "C"
