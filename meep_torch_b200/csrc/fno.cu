// FNO channel mixes on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// The pointwise (1 x 1) layers of the cfg5 Fourier neural operator are GEMMs over
// pixels: for image b and pixel p, z[b, o, p] = sum_i W[o, i] x[b, i, p] (+ bias[o]
// + s[b, o, p], the spectral branch), y = GELU(z). Activations are NCHW float32;
// the tensor cores take BF16 operands and accumulate in FP32 (TMEM).
//
// One CTA = 4 warps. A tile is 128 pixels (M = 128): thread t owns pixel t and
// TMEM lane t (warp w reads lanes 32w .. 32w+31). The operands are staged by the
// threads into shared memory in the K-major, no-swizzle canonical layout (core
// matrices of 8 rows x 16 bytes; LBO = 128 B between the two K halves of one
// MMA, SBO between 8-row groups), one elected thread issues K/16
// tcgen05.mma.kind::f16 into TMEM and commits to an mbarrier, and the epilogue
// reads the accumulator back with tcgen05.ld. Every mbarrier wait is bounded:
// on expiry the kernel records MTB_DEVICE_TIMEOUT (mtb_fno_status), waits once
// more with a bound, frees its TMEM and returns.
//
//   k_fno_mix   forward: A = x^T (pixels x C_in), B = W (C_out x C_in, K-major);
//               epilogue + bias + s, optional store of z, GELU.
//   k_fno_dx    backward to x: dz = dy * GELU'(z) formed while staging A (and
//               stored for dW), B = W^T; dx = dz^T W.
//   k_fno_dw    backward to W: K = pixels. A = dz rows (C_out, zero-padded to
//               128), B = x rows (C_in); partial sums of a CTA's pixel range
//               accumulate in TMEM and are added into dW with atomicAdd.
#include <cuda_bf16.h>

#include <algorithm>

#include "mtb_common.cuh"

namespace mtb {
namespace {

constexpr int FNO_THREADS = 128;
// Dynamic shared memory per CTA: at least what the operands need, and at least a
// floor that bounds the CTAs an SM can hold (233472 bytes of shared memory, 1 KB
// reserved per CTA) so that their TMEM never exceeds the SM's 512 columns and
// tcgen05.alloc never waits on another CTA: 64 columns -> 29 KB floor (at most 7 CTAs,
// 448 columns); 128 columns -> 58 KB (at most 3 CTAs, 384 columns).
constexpr int smem_bytes(int need, int ncols) {
    return need > (ncols <= 64 ? 29 * 1024 : 58 * 1024) ? need
                                                        : (ncols <= 64 ? 29 * 1024 : 58 * 1024);
}
constexpr int tmem_cols(int n) { return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : 256; }
constexpr long long FNO_SPIN = 1LL << 24;        // polls of one mbarrier wait

__device__ int g_fno_err;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// byte offset of element (row, k) in a K-major no-swizzle tile whose 8-row groups
// are `sbo` bytes apart
__device__ __forceinline__ uint32_t kmaj(int row, int k, int sbo) {
    return (uint32_t)((row >> 3) * sbo + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor (sm100): start, LBO, SBO in 16-byte units,
// version 1, no swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D f32, A and B bf16, both K-major, M x N
constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db,
                                          uint32_t idesc, uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z),
          "r"(z));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void bar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// bounded wait for the phase `parity` of `bar` to complete
__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (long long it = 0; it < FNO_SPIN; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 16 consecutive FP32 accumulator columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// warp 0 allocates `ncols` TMEM columns; the base address lands in *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ void st_shared16(uint32_t addr, uint32_t a, uint32_t b, uint32_t c,
                                            uint32_t d) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c),
                 "r"(d)
                 : "memory");
}

// GELU with the exact erf form (torch.nn.functional.gelu, approximate='none')
__device__ __forceinline__ float gelu(float z) {
    return 0.5f * z * (1.f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.f + erff(z * 0.70710678118654752f)) +
           z * 0.39894228040143268f * expf(-0.5f * z * z);
}

struct alignas(8) FnoShared {
    uint64_t bar;
    uint32_t tmem;
    int ok;
};

// Common skeleton of k_fno_mix / k_fno_dx: W-derived B operand staged once, then a
// grid-stride loop over (image, 128-pixel tile). KIN = K (reduction width),
// NOUT = N (output channels of this GEMM).
template <int KIN, int NOUT, bool DX>
__global__ void __launch_bounds__(FNO_THREADS, 1)
    k_fno_pointwise(const float *__restrict__ src, const float *__restrict__ zin,
                    const float *__restrict__ W, const float *__restrict__ bias,
                    const float *__restrict__ s, float *__restrict__ out,
                    float *__restrict__ aux, int batch, long long P, int act) {
    static_assert(KIN % 16 == 0 && NOUT % 16 == 0 && NOUT >= 16 && NOUT <= 256, "shape");
    extern __shared__ __align__(1024) unsigned char smem[];
    constexpr int SBO_A = (KIN / 8) * 128;
    constexpr int SBO_B = (KIN / 8) * 128;
    constexpr int A_BYTES = 128 * KIN * 2;
    unsigned char *sA = smem;
    unsigned char *sB = smem + A_BYTES;
    FnoShared *sh = reinterpret_cast<FnoShared *>(smem + A_BYTES + NOUT * KIN * 2);
    const int t = threadIdx.x, warp = t >> 5;
    constexpr uint32_t NCOLS = tmem_cols(NOUT);

    // B operand: forward B[n=o][k=i] = W[o, i] (W is C_out x C_in);
    // dx        B[n=i][k=o] = W[o, i]  (here KIN = C_out, NOUT = C_in)
    for (int q = t; q < NOUT * KIN / 8; q += FNO_THREADS) {
        const int n = q / (KIN / 8), kc = (q % (KIN / 8)) * 8;
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            v[j] = DX ? W[(long long)(kc + j) * NOUT + n] : W[(long long)n * KIN + kc + j];
        st_shared16(smem_u32(sB) + kmaj(n, kc, SBO_B), pack_bf16(v[0], v[1]),
                    pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
    }
    if (t == 0) {
        bar_init(&sh->bar);
        sh->ok = 1;
    }
    if (warp == 0) tmem_alloc(&sh->tmem, NCOLS);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = sh->tmem;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    constexpr uint32_t IDESC = idesc_bf16(128, NOUT);
    const long long tiles_per_img = (P + 127) / 128;
    const long long n_tiles = tiles_per_img * batch;
    uint32_t parity = 0;

    for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int b = (int)(tile / tiles_per_img);
        const long long p = (tile % tiles_per_img) * 128 + t;
        const bool valid = p < P;
        // A[m = pixel][k]: forward x[b, k, p]; dx dz[b, k, p] = dy * GELU'(z).
        // 32 channels per pass: all loads first (32 or 64 in flight per thread),
        // then the transform and the four 16-byte shared stores.
#pragma unroll 1
        for (int k0 = 0; k0 < KIN; k0 += 32) {
            float v[32], zz[DX ? 32 : 1];
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const long long g = ((long long)b * KIN + k0 + j) * P + p;
                v[j] = valid ? src[g] : 0.f;
                if (DX) zz[DX ? j : 0] = (valid && act) ? zin[g] : 0.f;
            }
            if (DX) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    if (act) v[j] *= gelu_grad(zz[DX ? j : 0]);
                    if (aux && valid) aux[((long long)b * KIN + k0 + j) * P + p] = v[j];
                }
            }
#pragma unroll
            for (int c = 0; c < 4; ++c)
                st_shared16(smem_u32(sA) + kmaj(t, k0 + 8 * c, SBO_A),
                            pack_bf16(v[8 * c], v[8 * c + 1]), pack_bf16(v[8 * c + 2], v[8 * c + 3]),
                            pack_bf16(v[8 * c + 4], v[8 * c + 5]),
                            pack_bf16(v[8 * c + 6], v[8 * c + 7]));
        }
        fence_async_smem();
        __syncthreads();
        // the spectral term of this pixel, fetched while the tensor cores run
        constexpr bool PRE = !DX && NOUT <= 64;
        float sp[PRE ? NOUT : 1];
        if (PRE) {
#pragma unroll
            for (int o = 0; o < (PRE ? NOUT : 1); ++o)
                sp[o] = (s && valid) ? s[((long long)b * NOUT + o) * P + p] : 0.f;
        }
        if (t == 0) {
            fence_after();
#pragma unroll
            for (int ks = 0; ks < KIN / 16; ++ks)
                umma_bf16(tmem, sdesc(smem_u32(sA) + ks * 256, 128, SBO_A),
                          sdesc(smem_u32(sB) + ks * 256, 128, SBO_B), IDESC, ks > 0);
            umma_commit(&sh->bar);
            if (!bar_wait(&sh->bar, parity)) {
                atomicExch(&g_fno_err, 1);
                bar_wait(&sh->bar, parity);
                sh->ok = 0;
            }
        }
        parity ^= 1;
        __syncthreads();
        if (!sh->ok) break;
        fence_after();
#pragma unroll
        for (int g = 0; g < NOUT; g += 16) {
            float v[16];
            tmem_ld16(lane_base + g, v);
            if (!valid) continue;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int o = g + j;
                const long long gi = ((long long)b * NOUT + o) * P + p;
                float z = v[j];
                if (!DX) {
                    if (bias) z += bias[o];
                    if (PRE) z += sp[(PRE ? o : 0)];
                    else if (s) z += s[gi];
                    if (aux) aux[gi] = z;
                    if (act) z = gelu(z);
                }
                out[gi] = z;
            }
        }
        fence_before();
        __syncthreads();
    }
    fence_after();
    __syncthreads();
    if (warp == 0) tmem_free(tmem, NCOLS);
}

// dW[o, i] += sum over this CTA's (image, 128-pixel) tiles of dz[b, o, p] x[b, i, p].
// A rows: C_out (zero-padded to 128); B rows: C_in; K = 128 pixels per tile.
template <int COUT, int CIN>
__global__ void __launch_bounds__(FNO_THREADS, 1)
    k_fno_dw(const float *__restrict__ dz, const float *__restrict__ x, float *__restrict__ dW,
             int batch, long long P) {
    static_assert(COUT <= 128 && CIN % 16 == 0 && CIN <= 256, "shape");
    extern __shared__ __align__(1024) unsigned char smem[];
    constexpr int KT = 128;                       // pixels per tile
    constexpr int SBO = (KT / 8) * 128;            // 2048 B
    constexpr int A_BYTES = 128 * KT * 2;
    unsigned char *sA = smem;
    unsigned char *sB = smem + A_BYTES;
    FnoShared *sh = reinterpret_cast<FnoShared *>(smem + A_BYTES + CIN * KT * 2);
    const int t = threadIdx.x, warp = t >> 5;
    constexpr uint32_t NCOLS = tmem_cols(CIN);
    // rows COUT .. 127 of A stay zero
    for (int q = t; q < (128 - COUT) * KT / 8; q += FNO_THREADS) {
        const int r = COUT + q / (KT / 8), kc = (q % (KT / 8)) * 8;
        st_shared16(smem_u32(sA) + kmaj(r, kc, SBO), 0u, 0u, 0u, 0u);
    }
    if (t == 0) {
        bar_init(&sh->bar);
        sh->ok = 1;
    }
    if (warp == 0) tmem_alloc(&sh->tmem, NCOLS);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = sh->tmem;
    const long long tiles_per_img = (P + KT - 1) / KT;
    const long long n_tiles = tiles_per_img * batch;
    const long long per = (n_tiles + gridDim.x - 1) / gridDim.x;
    const long long t0 = (long long)blockIdx.x * per;
    const long long t1 = t0 + per < n_tiles ? t0 + per : n_tiles;
    constexpr uint32_t IDESC = idesc_bf16(128, CIN);
    uint32_t parity = 0;
    bool any = false;
    for (long long tile = t0; tile < t1; ++tile) {
        const int b = (int)(tile / tiles_per_img);
        const long long p0 = (tile % tiles_per_img) * KT;
        // 8 consecutive pixels of one row per chunk (float4 pairs; P % 8 == 0)
#pragma unroll 4
        for (int q = t; q < (COUT + CIN) * (KT / 8); q += FNO_THREADS) {
            const int row = q / (KT / 8), kc = (q % (KT / 8)) * 8;
            const bool isA = row < COUT;
            const float *base = isA ? dz + ((long long)b * COUT + row) * P
                                    : x + ((long long)b * CIN + (row - COUT)) * P;
            float4 u = make_float4(0.f, 0.f, 0.f, 0.f), w = u;
            if (p0 + kc < P) {
                u = *reinterpret_cast<const float4 *>(base + p0 + kc);
                w = *reinterpret_cast<const float4 *>(base + p0 + kc + 4);
            }
            const uint32_t dst = isA ? smem_u32(sA) + kmaj(row, kc, SBO)
                                     : smem_u32(sB) + kmaj(row - COUT, kc, SBO);
            st_shared16(dst, pack_bf16(u.x, u.y), pack_bf16(u.z, u.w), pack_bf16(w.x, w.y),
                        pack_bf16(w.z, w.w));
        }
        fence_async_smem();
        __syncthreads();
        if (t == 0) {
            fence_after();
#pragma unroll
            for (int ks = 0; ks < KT / 16; ++ks)
                umma_bf16(tmem, sdesc(smem_u32(sA) + ks * 256, 128, SBO),
                          sdesc(smem_u32(sB) + ks * 256, 128, SBO), IDESC,
                          (any || ks > 0) ? 1u : 0u);
            umma_commit(&sh->bar);
            if (!bar_wait(&sh->bar, parity)) {
                atomicExch(&g_fno_err, 1);
                bar_wait(&sh->bar, parity);
                sh->ok = 0;
            }
        }
        parity ^= 1;
        any = true;
        __syncthreads();
        if (!sh->ok) break;
    }
    fence_after();
    if (any && sh->ok && warp * 32 < COUT) {
        const int o = warp * 32 + (t & 31);
        const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int g = 0; g < CIN; g += 16) {
            float v[16];
            tmem_ld16(lane_base + g, v);
            if (o < COUT) {
#pragma unroll
                for (int j = 0; j < 16; ++j) atomicAdd(dW + (long long)o * CIN + g + j, v[j]);
            }
        }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) tmem_free(tmem, NCOLS);
}

int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            n = 148;
    }
    return n;
}

// shared memory a launch of each kernel requests (operands + barrier block)
template <int KIN, int NOUT>
constexpr int pointwise_smem() {
    return smem_bytes(128 * KIN * 2 + NOUT * KIN * 2 + 64, tmem_cols(NOUT));
}
template <int CIN>
constexpr int dw_smem() {
    return smem_bytes(128 * 128 * 2 + CIN * 128 * 2 + 64, tmem_cols(CIN));
}

// sets the kernel's shared-memory limit and returns its grid: one wave of the CTAs
// the SMs hold at once (by registers, shared memory and TMEM columns), at most one
// per tile. The residency is computed here from the kernel's register count:
// cudaOccupancyMaxActiveBlocksPerMultiprocessor reported one CTA per SM for these
// kernels where two and more are resident.
template <class K>
int prepare(K kern, int smem, int ncols, long long tiles, int *grid) {
    MTB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    cudaFuncAttributes fa;
    MTB_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    const int regs_warp = ((fa.numRegs * 32 + 255) / 256) * 256;     // per-warp granularity
    const int by_regs = 65536 / (regs_warp * (FNO_THREADS / 32));
    const int by_smem = 233472 / (smem + (int)fa.sharedSizeBytes + 1024);
    const int by_tmem = 512 / ncols;
    const int per_sm = std::max(1, std::min(std::min(by_regs, by_smem), by_tmem));
    *grid = (int)std::min<long long>(tiles, (long long)per_sm * sm_count());
    return MTB_OK;
}

int check_shape(int batch, int cin, int cout, long long P) {
    if (batch < 1 || P < 1)
        return fail(MTB_INVALID_ARG, "fno: batch=%d pixels=%lld must be positive", batch, P);
    if (P % 8)
        return fail(MTB_INVALID_ARG, "fno: pixels=%lld must be a multiple of 8", P);
    if (cin != 64 || (cout != 64 && cout != 128))
        return fail(MTB_UNSUPPORTED, "fno: channel mix %d -> %d (built: 64 -> 64, 64 -> 128)",
                    cin, cout);
    return MTB_OK;
}

int aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace
}  // namespace mtb

using namespace mtb;

extern "C" {

int mtb_fno_mix(const float *x, const float *w, const float *bias, const float *s, float *y,
                float *z, int32_t batch, int32_t cin, int32_t cout, int64_t pixels,
                int32_t act, void *stream) {
    int rc;
    if ((rc = check_shape(batch, cin, cout, pixels))) return rc;
    if (!x || !w || !y) return fail(MTB_INVALID_ARG, "fno_mix: null x, w or y");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long tiles = (long long)batch * ((pixels + 127) / 128);
    int grid = 0;
    if (cout == 64) {
        constexpr int sm = pointwise_smem<64, 64>();
        if ((rc = prepare(k_fno_pointwise<64, 64, false>, sm, 64, tiles, &grid))) return rc;
        k_fno_pointwise<64, 64, false><<<grid, FNO_THREADS, sm, st>>>(
            x, nullptr, w, bias, s, y, z, batch, pixels, act);
    } else {
        constexpr int sm = pointwise_smem<64, 128>();
        if ((rc = prepare(k_fno_pointwise<64, 128, false>, sm, 128, tiles, &grid))) return rc;
        k_fno_pointwise<64, 128, false><<<grid, FNO_THREADS, sm, st>>>(
            x, nullptr, w, bias, s, y, z, batch, pixels, act);
    }
    MTB_CHECK_LAUNCH();
    return MTB_OK;
}

int mtb_fno_mix_dx(const float *dy, const float *z, const float *w, float *dz, float *dx,
                   int32_t batch, int32_t cin, int32_t cout, int64_t pixels, int32_t act,
                   void *stream) {
    int rc;
    if ((rc = check_shape(batch, cin, cout, pixels))) return rc;
    if (!dy || !w || !dx || (act && !z)) return fail(MTB_INVALID_ARG, "fno_mix_dx: null input");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long tiles = (long long)batch * ((pixels + 127) / 128);
    int grid = 0;
    if (cout == 64) {
        constexpr int sm = pointwise_smem<64, 64>();
        if ((rc = prepare(k_fno_pointwise<64, 64, true>, sm, 64, tiles, &grid))) return rc;
        k_fno_pointwise<64, 64, true><<<grid, FNO_THREADS, sm, st>>>(
            dy, z, w, nullptr, nullptr, dx, dz, batch, pixels, act);
    } else {
        constexpr int sm = pointwise_smem<128, 64>();
        if ((rc = prepare(k_fno_pointwise<128, 64, true>, sm, 64, tiles, &grid))) return rc;
        k_fno_pointwise<128, 64, true><<<grid, FNO_THREADS, sm, st>>>(
            dy, z, w, nullptr, nullptr, dx, dz, batch, pixels, act);
    }
    MTB_CHECK_LAUNCH();
    return MTB_OK;
}

int mtb_fno_mix_dw(const float *dz, const float *x, float *dw, int32_t batch, int32_t cin,
                   int32_t cout, int64_t pixels, void *stream) {
    int rc;
    if ((rc = check_shape(batch, cin, cout, pixels))) return rc;
    if (!dz || !x || !dw) return fail(MTB_INVALID_ARG, "fno_mix_dw: null input");
    if (!aligned16(dz) || !aligned16(x))
        return fail(MTB_INVALID_ARG, "fno_mix_dw: dz and x must be 16-byte aligned");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long tiles = (long long)batch * ((pixels + 127) / 128);
    int grid = 0;
    constexpr int sm = dw_smem<64>();
    if (cout == 64) {
        if ((rc = prepare(k_fno_dw<64, 64>, sm, 64, tiles, &grid))) return rc;
        k_fno_dw<64, 64><<<grid, FNO_THREADS, sm, st>>>(dz, x, dw, batch, pixels);
    } else {
        if ((rc = prepare(k_fno_dw<128, 64>, sm, 64, tiles, &grid))) return rc;
        k_fno_dw<128, 64><<<grid, FNO_THREADS, sm, st>>>(dz, x, dw, batch, pixels);
    }
    MTB_CHECK_LAUNCH();
    return MTB_OK;
}

int mtb_fno_status(void *stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    MTB_CUDA_TRY(cudaStreamSynchronize(st));
    int flag = 0;
    MTB_CUDA_TRY(cudaMemcpyFromSymbol(&flag, g_fno_err, sizeof(int)));
    if (flag) {
        const int zero = 0;
        MTB_CUDA_TRY(cudaMemcpyToSymbol(g_fno_err, &zero, sizeof(int)));
        return fail(MTB_DEVICE_TIMEOUT, "fno: a bounded tensor-core wait expired");
    }
    return MTB_OK;
}

}  // extern "C"
