// Error state, launch counter, layout kernels and the DFT ring contraction.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <vector>

#include "mtb_common.cuh"

namespace mtb {

static thread_local char g_err[1024] = "";
static std::atomic<int64_t> g_launches{0};

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

void count_launch(int64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// ------------------------------------------------------------ launch timer

int LaunchTimer::begin(cudaStream_t st, int k) {
    if (!on) return MTB_OK;
    while (pool.size() < used + 2) {
        cudaEvent_t e;
        MTB_CUDA_TRY(cudaEventCreate(&e));
        pool.push_back(e);
    }
    kind.resize(pool.size() / 2 + 1);
    kind[used / 2] = k;
    MTB_CUDA_TRY(cudaEventRecord(pool[used], st));
    return MTB_OK;
}

int LaunchTimer::end(cudaStream_t st) {
    if (!on) return MTB_OK;
    MTB_CUDA_TRY(cudaEventRecord(pool[used + 1], st));
    used += 2;
    return MTB_OK;
}

int LaunchTimer::collect() {
    if (!on || used == 0) return MTB_OK;
    MTB_CUDA_TRY(cudaEventSynchronize(pool[used - 1]));
    for (size_t i = 0; i < used; i += 2) {
        float t = 0.f;
        MTB_CUDA_TRY(cudaEventElapsedTime(&t, pool[i], pool[i + 1]));
        ms[kind[i / 2]] += t;
        count[kind[i / 2]] += 1;
    }
    used = 0;
    return MTB_OK;
}

void LaunchTimer::release() {
    for (auto e : pool) cudaEventDestroy(e);
    pool.clear();
    used = 0;
}

// ------------------------------------------------------------ layout kernels

// Writes the whole box: the block [off, off+n) gets src, the rest zero.
__global__ void k_pack(const float *__restrict__ src, int64_t n0, int64_t n1, int64_t n2,
                       int64_t s0, int64_t s1, float *__restrict__ box, int64_t bn0,
                       int64_t bn1, int64_t bn2, int64_t b0, int64_t b1, int64_t o0,
                       int64_t o1, int64_t o2) {
    const int64_t total = bn0 * bn1 * bn2;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = idx % bn2;
        const int64_t r = idx / bn2;
        const int64_t j = r % bn1;
        const int64_t i = r / bn1;
        const int64_t si = i - o0, sj = j - o1, sk = k - o2;
        float v = 0.f;
        if (si >= 0 && si < n0 && sj >= 0 && sj < n1 && sk >= 0 && sk < n2)
            v = src[si * s0 + sj * s1 + sk];
        box[i * b0 + j * b1 + k] = v;
    }
}

__global__ void k_unpack(const float *__restrict__ box, int64_t n0, int64_t n1, int64_t n2,
                         int64_t b0, int64_t b1, int64_t o0, int64_t o1, int64_t o2,
                         float *__restrict__ dst, int64_t s0, int64_t s1) {
    const int64_t total = n0 * n1 * n2;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = idx % n2;
        const int64_t r = idx / n2;
        const int64_t j = r % n1;
        const int64_t i = r / n1;
        dst[i * s0 + j * s1 + k] = box[(i + o0) * b0 + (j + o1) * b1 + (k + o2)];
    }
}

__global__ void k_unpack_ratio(const float *__restrict__ box, const float *__restrict__ den,
                               int64_t n0, int64_t n1, int64_t n2, int64_t b0, int64_t b1,
                               int64_t o0, int64_t o1, int64_t o2, float *__restrict__ dst,
                               int64_t s0, int64_t s1) {
    const int64_t total = n0 * n1 * n2;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = idx % n2;
        const int64_t r = idx / n2;
        const int64_t j = r % n1;
        const int64_t i = r / n1;
        const int64_t b = (i + o0) * b0 + (j + o1) * b1 + (k + o2);
        dst[i * s0 + j * s1 + k] = box[b] / den[b];
    }
}

__global__ void k_count_outside(const float *__restrict__ x, int64_t n0, int64_t n1, int64_t s0,
                                const uint8_t *__restrict__ a0, const uint8_t *__restrict__ a1,
                                unsigned long long *count) {
    const int64_t total = n0 * n1;
    unsigned long long c = 0;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = idx % n1, i = idx / n1;
        const bool act = (a0 && a0[i]) || (a1 && a1[j]);
        if (!act && x[i * s0 + j] != 0.f) ++c;
    }
    if (c) atomicAdd(count, c);
}

static int grid_for(int64_t total, int threads = 256) {
    int64_t b = (total + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (int)b;
}

// ------------------------------------------------------------ DFT contraction

constexpr int KMAX = 64;       // deepest ring supported by the contraction
constexpr int CT = 256;        // channels per contraction block

// One block folds CT channels of one region (region of the block from a
// per-block table). Phase values of the region's (group, toff) are staged
// in shared memory, sP[s * nf + f] = (Re, Im); each thread keeps NFC
// frequencies of its channel in registers and streams its n ring samples.
constexpr int NFC = 4;
constexpr int KFULL = 32;      // ring depth with a fully unrolled contraction (the default)
__global__ void __launch_bounds__(CT, 4) k_dft_contract(
    const mtb_dft_region *__restrict__ regions, const int *__restrict__ blk_region,
    const int64_t *__restrict__ blk_start, const int *__restrict__ group_nf,
    const int *__restrict__ group_off, int total_nf, const float *__restrict__ phase, int row0,
    int n, const float *__restrict__ ring, int64_t slot_elems) {
    extern __shared__ float2 sP[];
    const int64_t b = blockIdx.x;
    const int rg = blk_region[b];
    const mtb_dft_region R = regions[rg];
    const int nf = group_nf[R.group];
    const int foff = group_off[R.group];
    const int sel = (R.toff == 2) ? 2 : 0;
    for (int e = threadIdx.x; e < n * nf; e += CT) {
        const int s = e / nf, f = e - s * nf;
        const float *p = phase + ((int64_t)(row0 + s) * total_nf + foff + f) * 4 + sel;
        sP[e] = make_float2(p[0], p[1]);
    }
    __syncthreads();
    const int64_t ch = (b - blk_start[rg]) * CT + threadIdx.x;
    const int64_t nch = (int64_t)R.rows * R.cols;
    if (ch >= nch) return;
    // frequencies [fa, fb) of this block row (small channel counts split the
    // frequency loop over gridDim.y block rows; each sum is formed as without it)
    const int per = (nf + gridDim.y - 1) / gridDim.y;
    const int fa = blockIdx.y * per, fb = min(nf, fa + per);
    if (fa >= fb) return;
    const int r = (int)(ch / R.cols), c = (int)(ch - (int64_t)r * R.cols);
    const float *xa = ring + R.ring_a + (int64_t)r * R.ring_pitch + c;
    const float *xb = (R.ring_b >= 0) ? ring + R.ring_b + (int64_t)r * R.ring_pitch + c : nullptr;
    float *acc = R.acc;
    const int64_t base = (int64_t)r * R.acc_pitch + c;
    if (n == KFULL) {
        // a whole ring: every sample of the channel in flight at once
        float x[KFULL];
#pragma unroll
        for (int s = 0; s < KFULL; ++s) x[s] = __ldg(xa + s * slot_elems);
        if (xb) {
#pragma unroll
            for (int s = 0; s < KFULL; ++s) x[s] = 0.5f * (x[s] + __ldg(xb + s * slot_elems));
        }
        for (int f = fa; f < fb; ++f) {
            float re = 0.f, im = 0.f;
#pragma unroll
            for (int s = 0; s < KFULL; ++s) {
                const float2 p = sP[s * nf + f];
                re = fmaf(p.x, x[s], re);
                im = fmaf(p.y, x[s], im);
            }
            acc[R.re_off + f * R.f_stride + base] += re;
            acc[R.im_off + f * R.f_stride + base] += im;
        }
        return;
    }
    for (int f0 = fa; f0 < fb; f0 += NFC) {
        float *pr[NFC], *pi[NFC];
        float re[NFC], im[NFC];
#pragma unroll
        for (int q = 0; q < NFC; ++q) {
            const int f = min(f0 + q, fb - 1);
            pr[q] = acc + R.re_off + f * R.f_stride + base;
            pi[q] = acc + R.im_off + f * R.f_stride + base;
            re[q] = 0.f;
            im[q] = 0.f;
        }
#pragma unroll 4
        for (int s = 0; s < n; ++s) {
            float x = xa[s * slot_elems];
            if (xb) x = 0.5f * (x + xb[s * slot_elems]);
            const float2 *ps = sP + s * nf + f0;
#pragma unroll
            for (int q = 0; q < NFC; ++q) {
                if (f0 + q < fb) {
                    const float2 p = ps[q];
                    re[q] = fmaf(p.x, x, re[q]);
                    im[q] = fmaf(p.y, x, im[q]);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NFC; ++q) {
            if (f0 + q < fb) {
                *pr[q] += re[q];
                *pi[q] += im[q];
            }
        }
    }
}

// Transpose of k_dft_contract (the adjoint of DFT sampling): for ring slot
// s of the n staged steps, every channel of a region receives
//   sum_f Re P(s, f) acc_re[f, ch] + Im P(s, f) acc_im[f, ch]
// (acc = d J / d accumulator), split 1/2 : 1/2 onto ring_a / ring_b where
// the forward averaged two samples. Regions may share ring elements, so the
// ring (zeroed by the caller) is accumulated atomically.
__global__ void __launch_bounds__(CT) k_dft_expand(
    const mtb_dft_region *__restrict__ regions, const int *__restrict__ blk_region,
    const int64_t *__restrict__ blk_start, const int *__restrict__ group_nf,
    const int *__restrict__ group_off, int total_nf, const float *__restrict__ phase, int row0,
    int n, float *__restrict__ ring, int64_t slot_elems) {
    extern __shared__ float2 sP[];
    const int64_t b = blockIdx.x;
    const int rg = blk_region[b];
    const mtb_dft_region R = regions[rg];
    const int nf = group_nf[R.group];
    const int foff = group_off[R.group];
    const int sel = (R.toff == 2) ? 2 : 0;
    for (int e = threadIdx.x; e < n * nf; e += CT) {
        const int s = e / nf, f = e - s * nf;
        const float *p = phase + ((int64_t)(row0 + s) * total_nf + foff + f) * 4 + sel;
        sP[e] = make_float2(p[0], p[1]);
    }
    __syncthreads();
    const int64_t ch = (b - blk_start[rg]) * CT + threadIdx.x;
    const int64_t nch = (int64_t)R.rows * R.cols;
    if (ch >= nch) return;
    const int r = (int)(ch / R.cols), c = (int)(ch - (int64_t)r * R.cols);
    float *xa = ring + R.ring_a + (int64_t)r * R.ring_pitch + c;
    float *xb = (R.ring_b >= 0) ? ring + R.ring_b + (int64_t)r * R.ring_pitch + c : nullptr;
    const float *acc = R.acc;
    const int64_t base = (int64_t)r * R.acc_pitch + c;
    for (int s = 0; s < n; ++s) {
        float g = 0.f;
        for (int f = 0; f < nf; ++f) {
            const float2 p = sP[s * nf + f];
            g = fmaf(p.x, __ldg(acc + R.re_off + f * R.f_stride + base), g);
            g = fmaf(p.y, __ldg(acc + R.im_off + f * R.f_stride + base), g);
        }
        if (xb) {
            atomicAdd(xa + s * slot_elems, 0.5f * g);
            atomicAdd(xb + s * slot_elems, 0.5f * g);
        } else {
            atomicAdd(xa + s * slot_elems, g);
        }
    }
}

int DftState::init(const mtb_dft_region *regions, int nreg, const mtb_phase_group *groups,
                   int ngrp, int64_t selems, int nslots) {
    n_regions = nreg;
    n_groups = ngrp;
    slot_elems = selems;
    slots = nslots;
    if (nslots < 1 || nslots > KMAX)
        return fail(MTB_INVALID_ARG, "ring_slots must be in [1, %d], got %d", KMAX, nslots);
    if (nreg < 0 || ngrp < 0) return fail(MTB_INVALID_ARG, "negative region/group count");
    if (nreg > 0 && (!regions || !groups)) return fail(MTB_INVALID_ARG, "null regions/groups");
    group_nf = (int *)calloc(ngrp + 1, sizeof(int));
    group_mode = (int *)calloc(ngrp + 1, sizeof(int));
    group_dt = (double *)calloc(ngrp + 1, sizeof(double));
    freq_off = (int *)calloc(ngrp + 1, sizeof(int));
    total_nf = 0;
    for (int g = 0; g < ngrp; ++g) {
        if (groups[g].nf < 1 || groups[g].nf > 256 || !groups[g].freqs)
            return fail(MTB_INVALID_ARG, "phase group %d: nf=%d out of [1,256] or null freqs", g,
                        groups[g].nf);
        if (groups[g].mode != 0 && groups[g].mode != 1)
            return fail(MTB_INVALID_ARG, "phase group %d: mode must be 0 or 1", g);
        group_nf[g] = groups[g].nf;
        group_mode[g] = groups[g].mode;
        group_dt[g] = groups[g].dt;
        freq_off[g] = total_nf;
        total_nf += groups[g].nf;
    }
    freqs_h = (double *)calloc(total_nf + 1, sizeof(double));
    for (int g = 0; g < ngrp; ++g)
        memcpy(freqs_h + freq_off[g], groups[g].freqs, sizeof(double) * groups[g].nf);
    regions_h = (mtb_dft_region *)calloc(nreg + 1, sizeof(mtb_dft_region));
    if (nreg) memcpy(regions_h, regions, sizeof(mtb_dft_region) * nreg);
    blk_start_h = (int *)calloc(nreg + 1, sizeof(int));
    std::vector<int64_t> bs(nreg + 1, 0);
    int64_t nb = 0;
    for (int r = 0; r < nreg; ++r) {
        const mtb_dft_region &R = regions[r];
        if (R.group < 0 || R.group >= ngrp)
            return fail(MTB_INVALID_ARG, "region %d: bad group %d", r, R.group);
        if (R.toff != 1 && R.toff != 2)
            return fail(MTB_INVALID_ARG, "region %d: toff must be 1 or 2", r);
        if (R.rows < 0 || R.cols < 0 || !R.acc)
            return fail(MTB_INVALID_ARG, "region %d: bad extent or null accumulator", r);
        if (R.ring_a < 0 || R.ring_a + (int64_t)(R.rows - 1) * R.ring_pitch + R.cols > selems ||
            (R.ring_b >= 0 && R.ring_b + (int64_t)(R.rows - 1) * R.ring_pitch + R.cols > selems))
            return fail(MTB_INVALID_ARG, "region %d: ring window outside the slot (%lld elems)", r,
                        (long long)selems);
        bs[r] = nb;
        nb += ((int64_t)R.rows * R.cols + CT - 1) / CT;
    }
    bs[nreg] = nb;
    n_blocks = nb;
    if (nb > 0x7fffffffLL) return fail(MTB_INVALID_ARG, "too many DFT channels");
    std::vector<int> br((size_t)nb + 1, 0);
    for (int r = 0; r < nreg; ++r)
        for (int64_t q = bs[r]; q < bs[r + 1]; ++q) br[q] = r;
    int rc;
    if ((rc = blk_region_d.ensure(sizeof(int) * (br.size())))) return rc;
    MTB_CUDA_TRY(cudaMemcpy(blk_region_d.p, br.data(), sizeof(int) * br.size(),
                            cudaMemcpyHostToDevice));
    if ((rc = regions_d.ensure(sizeof(mtb_dft_region) * (nreg + 1)))) return rc;
    if ((rc = blk_start_d.ensure(sizeof(int64_t) * (nreg + 1) + 2 * sizeof(int) * (ngrp + 1))))
        return rc;
    if (nreg) MTB_CUDA_TRY(cudaMemcpy(regions_d.p, regions, sizeof(mtb_dft_region) * nreg,
                                      cudaMemcpyHostToDevice));
    MTB_CUDA_TRY(cudaMemcpy(blk_start_d.p, bs.data(), sizeof(int64_t) * (nreg + 1),
                            cudaMemcpyHostToDevice));
    int *gd = reinterpret_cast<int *>(blk_start_d.as<int64_t>() + (nreg + 1));
    MTB_CUDA_TRY(cudaMemcpy(gd, group_nf, sizeof(int) * (ngrp + 1), cudaMemcpyHostToDevice));
    MTB_CUDA_TRY(cudaMemcpy(gd + (ngrp + 1), freq_off, sizeof(int) * (ngrp + 1),
                            cudaMemcpyHostToDevice));
    // the ring exists whenever samples are written (DFT regions or stacked probes)
    if (selems > 0 && (rc = ring_d.ensure(sizeof(float) * (size_t)selems * nslots))) return rc;
    return MTB_OK;
}

int DftState::upload_phases(int64_t t0, int k, cudaStream_t st) {
    if (n_regions == 0) return MTB_OK;
    const size_t n = (size_t)k * total_nf * 4;
    int rc;
    void *hp = nullptr;
    if ((rc = phase_h.acquire(n * sizeof(float), &hp))) return rc;
    if ((rc = phase_d.ensure(n * sizeof(float)))) return rc;
    float *P = static_cast<float *>(hp);
    const double two_pi = 2.0 * M_PI;
    for (int g = 0; g < n_groups; ++g) {
        const double dt = group_dt[g];
        const float dtf = (float)dt;
        for (int f = 0; f < group_nf[g]; ++f) {
            const double fr = freqs_h[freq_off[g] + f];
            const float wf = (float)two_pi * (float)fr;   // reference float32 w
            for (int s = 0; s < k; ++s) {
                float *p = P + ((size_t)s * total_nf + freq_off[g] + f) * 4;
                for (int h = 0; h < 2; ++h) {
                    const double tt = ((double)(t0 + s) + 0.5 * (h + 1)) * dt;
                    float c, sn;
                    if (group_mode[g] == 0) {
                        const double arg = two_pi * fr * tt;
                        c = (float)(dt * cos(arg));
                        sn = (float)(-dt * sin(arg));
                    } else {
                        const float arg = wf * (float)tt;
                        c = dtf * cosf(arg);
                        sn = dtf * -sinf(arg);
                    }
                    p[2 * h] = c;
                    p[2 * h + 1] = sn;
                }
            }
        }
    }
    MTB_CUDA_TRY(cudaMemcpyAsync(phase_d.p, P, n * sizeof(float), cudaMemcpyHostToDevice, st));
    return phase_h.queued(st);
}

int DftState::contract(int row0, int n, cudaStream_t st, LaunchTimer *tm,
                       const float *phase_base) {
    if (n_regions == 0 || n <= 0 || n_blocks == 0) return MTB_OK;
    int maxnf = 1;
    for (int g = 0; g < n_groups; ++g) maxnf = std::max(maxnf, group_nf[g]);
    const size_t smem = sizeof(float2) * (size_t)n * maxnf;
    static bool attr_set = false;
    if (!attr_set) {
        MTB_CUDA_TRY(cudaFuncSetAttribute(k_dft_contract,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          sizeof(float2) * KMAX * 256));
        attr_set = true;
    }
    const int *gd = reinterpret_cast<const int *>(blk_start_d.as<int64_t>() + (n_regions + 1));
    if (n_blocks > 0x7fffffffLL) return fail(MTB_INVALID_ARG, "too many contraction blocks");
    int rc;
    if (tm && (rc = tm->begin(st, 1))) return rc;
    // few channels: split every channel's frequencies over block rows (four or more
    // frequencies each) until the launch has about 2^17 threads
    const int64_t want = ((int64_t)1 << 17) / std::max<int64_t>(n_blocks * CT, 1);
    const int fsplit = (int)std::max<int64_t>(1, std::min<int64_t>(want, (maxnf + 3) / 4));
    k_dft_contract<<<dim3((unsigned)n_blocks, fsplit), CT, smem, st>>>(
        regions_d.as<mtb_dft_region>(), blk_region_d.as<int>(), blk_start_d.as<int64_t>(), gd,
        gd + (n_groups + 1), total_nf, phase_base ? phase_base : phase_d.as<float>(), row0, n,
        ring_d.as<float>(),
        slot_elems);
    MTB_CHECK_LAUNCH();
    if (tm && (rc = tm->end(st))) return rc;
    return MTB_OK;
}

int DftState::expand(int row0, int n, cudaStream_t st) {
    if (n <= 0) return MTB_OK;
    MTB_CUDA_TRY(cudaMemsetAsync(ring_d.p, 0, sizeof(float) * (size_t)slot_elems * n, st));
    if (n_regions == 0 || n_blocks == 0) return MTB_OK;
    int maxnf = 1;
    for (int g = 0; g < n_groups; ++g) maxnf = std::max(maxnf, group_nf[g]);
    const size_t smem = sizeof(float2) * (size_t)n * maxnf;
    static bool attr_set = false;
    if (!attr_set) {
        MTB_CUDA_TRY(cudaFuncSetAttribute(k_dft_expand, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          sizeof(float2) * KMAX * 256));
        attr_set = true;
    }
    const int *gd = reinterpret_cast<const int *>(blk_start_d.as<int64_t>() + (n_regions + 1));
    k_dft_expand<<<(unsigned)n_blocks, CT, smem, st>>>(
        regions_d.as<mtb_dft_region>(), blk_region_d.as<int>(), blk_start_d.as<int64_t>(), gd,
        gd + (n_groups + 1), total_nf, phase_d.as<float>(), row0, n, ring_d.as<float>(),
        slot_elems);
    MTB_CHECK_LAUNCH();
    return MTB_OK;
}

void DftState::release() {
    regions_d.release();
    blk_start_d.release();
    blk_region_d.release();
    phase_d.release();
    ring_d.release();
    phase_h.release();
    free(regions_h);
    free(group_nf);
    free(group_mode);
    free(group_dt);
    free(freqs_h);
    free(freq_off);
    free(blk_start_h);
    regions_h = nullptr;
    group_nf = group_mode = freq_off = blk_start_h = nullptr;
    group_dt = freqs_h = nullptr;
}

}  // namespace mtb

using namespace mtb;

extern "C" {

const char *mtb_last_error(void) { return g_err; }

int32_t mtb_abi_version(void) { return MTB_ABI_VERSION; }

int64_t mtb_launch_count(void) { return g_launches.load(); }

int64_t mtb_struct_size(int32_t which) {
    switch (which) {
        case 0: return sizeof(mtb_cells);
        case 1: return sizeof(mtb_line_sample);
        case 2: return sizeof(mtb_yee2d_struct);
        case 3: return sizeof(mtb_phase_group);
        case 4: return sizeof(mtb_dft_region);
        case 5: return sizeof(mtb_tuning);
        case 6: return sizeof(mtb_yee3d_struct);
        case 7: return sizeof(mtb_adj2d_buffers);
        case 8: return sizeof(mtb_adj3d_buffers);
        default: return -1;
    }
}

int mtb_pack(const float *src, int64_t n0, int64_t n1, int64_t n2, int64_t s0, int64_t s1,
             float *box, int64_t bn0, int64_t bn1, int64_t bn2, int64_t b0, int64_t b1,
             int64_t o0, int64_t o1, int64_t o2, void *stream) {
    if (!box || (!src && n0 * n1 * n2 > 0)) return fail(MTB_INVALID_ARG, "mtb_pack: null pointer");
    if (n0 < 0 || n1 < 0 || n2 < 0 || o0 < 0 || o1 < 0 || o2 < 0 || o0 + n0 > bn0 ||
        o1 + n1 > bn1 || o2 + n2 > bn2 || bn2 > b1 || bn1 * b1 > b0)
        return fail(MTB_INVALID_ARG, "mtb_pack: block (%lld,%lld,%lld)+(%lld,%lld,%lld) outside box "
                    "(%lld,%lld,%lld)", (long long)n0, (long long)n1, (long long)n2, (long long)o0,
                    (long long)o1, (long long)o2, (long long)bn0, (long long)bn1, (long long)bn2);
    const int64_t total = bn0 * bn1 * bn2;
    if (total == 0) return MTB_OK;
    k_pack<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(src, n0, n1, n2, s0, s1, box, bn0,
                                                               bn1, bn2, b0, b1, o0, o1, o2);
    MTB_CHECK_LAUNCH();
    return MTB_OK;
}

int mtb_unpack(const float *box, int64_t n0, int64_t n1, int64_t n2, int64_t b0, int64_t b1,
               int64_t o0, int64_t o1, int64_t o2, float *dst, int64_t s0, int64_t s1,
               void *stream) {
    const int64_t total = n0 * n1 * n2;
    if (total == 0) return MTB_OK;
    if (!box || !dst) return fail(MTB_INVALID_ARG, "mtb_unpack: null pointer");
    if (n0 < 0 || n1 < 0 || n2 < 0 || o0 < 0 || o1 < 0 || o2 < 0)
        return fail(MTB_INVALID_ARG, "mtb_unpack: negative extent");
    k_unpack<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(box, n0, n1, n2, b0, b1, o0, o1, o2,
                                                                 dst, s0, s1);
    MTB_CHECK_LAUNCH();
    return MTB_OK;
}

int mtb_unpack_ratio(const float *box, const float *den, int64_t n0, int64_t n1, int64_t n2,
                     int64_t b0, int64_t b1, int64_t o0, int64_t o1, int64_t o2, float *dst,
                     int64_t s0, int64_t s1, void *stream) {
    const int64_t total = n0 * n1 * n2;
    if (total == 0) return MTB_OK;
    if (!box || !den || !dst) return fail(MTB_INVALID_ARG, "mtb_unpack_ratio: null pointer");
    if (n0 < 0 || n1 < 0 || n2 < 0 || o0 < 0 || o1 < 0 || o2 < 0)
        return fail(MTB_INVALID_ARG, "mtb_unpack_ratio: negative extent");
    k_unpack_ratio<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(box, den, n0, n1, n2, b0, b1,
                                                                       o0, o1, o2, dst, s0, s1);
    MTB_CHECK_LAUNCH();
    return MTB_OK;
}

int mtb_count_outside(const float *x, int64_t n0, int64_t n1, int64_t s0, const uint8_t *a0,
                      const uint8_t *a1, int64_t *count_dev, void *stream) {
    if (!x || !count_dev) return fail(MTB_INVALID_ARG, "mtb_count_outside: null pointer");
    const int64_t total = n0 * n1;
    MTB_CUDA_TRY(cudaMemsetAsync(count_dev, 0, sizeof(int64_t), (cudaStream_t)stream));
    if (total == 0) return MTB_OK;
    k_count_outside<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(
        x, n0, n1, s0, a0, a1, reinterpret_cast<unsigned long long *>(count_dev));
    MTB_CHECK_LAUNCH();
    return MTB_OK;
}

}  // extern "C"
