// Kernels of the learned preconditioner's convolutional network (a U-Net
// over [gradient, illumination, Vp, Vs] images), sm_100a:
//
//  * k_conv_kmajor  3x3 convolution (stride 1, zero padding 1) as an
//    implicit GEMM on the tcgen05 tensor cores: M = 128 pixels of one CTA,
//    N = output channels, K = 9 taps x input channels.  Operand tiles are
//    4-D / 3-D TMA boxes of the NHWC activation (shifted by the tap; the
//    zero fill of out-of-range boxes is the padding) and of the weights,
//    in the swizzled K-major layout; a 4-stage mbarrier pipeline feeds one
//    MMA-issuing thread; FP32 accumulators live in tensor memory; the
//    epilogue adds the bias and applies ReLU, or (input gradient) masks by a
//    ReLU output, and stores BF16 NHWC with any channel stride / offset.
//    The same kernel computes the input gradient with the tap-flipped,
//    transposed weights.
//  * k_conv_wgrad   weight gradient dW[tap][co][ci] = sum_p dz[p][co] x[p+tap][ci]
//    as a GEMM with M = output channels, N = input channels, K = pixels,
//    both operands MN-major (channels contiguous in NHWC), split over
//    pixel ranges with FP32 atomic accumulation.
//  * plain kernels for input packing, 2x2 average pooling, nearest 2x
//    upsampling into concatenation buffers, their gradients, the 1x1 output
//    head with its masked mean-square loss, bias gradients, weight packing
//    and the Adam update.
//
// Every mbarrier wait is bounded; a wait that gives up raises an error flag
// that the host reads.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <cstring>
#include <string>

#include "../../include/stfwi.h"
#include "../../include/stfwi_nn.h"
#include "tma.cuh"
#include "umma.cuh"

namespace stfwi {
namespace nn {

constexpr int CONV_THREADS = 128;
constexpr int STAGES = 4;
constexpr uint32_t NN_WAIT = 1u << 22;   // mbarrier polls before a wait gives up
constexpr int WG_PIX = 64;                // pixels per k-block of the weight gradient

struct ConvGeo {
    int n, h, w;          // images and spatial size (input = output size)
    int cin, cout;        // channels of the input tensor (contiguous NHWC) and of the output
    int kc;               // input channels per k-block: 16, 32 or 64 (the swizzle atom is 2*kc bytes)
    int bn;               // output channels per CTA (multiple of 16, <= 128)
    int bw, bh;           // pixel box of a CTA, bw * bh = 128
    int y_cstride, y_coff;
    int act;              // 0 none, 1 ReLU
    int m_cstride, m_coff;  // mask (input gradient): multiply by [mask > 0]
};

struct WgradGeo {
    int n, h, w;
    int cout, cin;        // channels of dz (M side) and of x (N side)
    int ae_a, ae_b;       // swizzle atom width in elements along M and along N
    int bn;               // input channels per CTA (multiple of ae_b, <= 128)
    int ci_tiles;
    int chunks, chunks_per_split;  // 64-pixel row chunks in total and per CTA
};

__host__ __device__ inline uint32_t tmem_cols_for(int n)
{
    uint32_t c = 32;
    while (c < (uint32_t)n) c <<= 1;
    return c;
}

__device__ __forceinline__ uint8_t *align1024(uint8_t *p)
{
    const uint32_t a = smem_u32(p);
    return p + (((a + 1023u) & ~1023u) - a);
}

__device__ __forceinline__ void store_bf16x16(__nv_bfloat16 *dst, const float (&v)[16])
{
    uint4 q[2];
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(q);
#pragma unroll
    for (int i = 0; i < 8; ++i) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    reinterpret_cast<uint4 *>(dst)[0] = q[0];
    reinterpret_cast<uint4 *>(dst)[1] = q[1];
}

__device__ __forceinline__ void load_bf16x16(const __nv_bfloat16 *src, float (&v)[16])
{
    uint4 q[2];
    q[0] = reinterpret_cast<const uint4 *>(src)[0];
    q[1] = reinterpret_cast<const uint4 *>(src)[1];
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(q);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float2 f = __bfloat1622float2(h[i]);
        v[2 * i] = f.x;
        v[2 * i + 1] = f.y;
    }
}

extern __shared__ uint8_t nn_smem[];

// ------------------------------------------------------------------ conv (K-major)

__global__ void __launch_bounds__(CONV_THREADS, 1)
    k_conv_kmajor(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmW, ConvGeo g,
                  const float *__restrict__ bias, const __nv_bfloat16 *__restrict__ mask,
                  __nv_bfloat16 *__restrict__ y, int *err)
{
    const uint32_t aw = 2u * g.kc;
    const uint32_t a_bytes = 128u * aw;                      // multiple of 1024
    const uint32_t b_bytes = (uint32_t)g.bn * aw;
    const uint32_t st_bytes = a_bytes + ((b_bytes + 1023u) & ~1023u);
    uint8_t *base = align1024(nn_smem);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + STAGES * st_bytes);
    uint64_t *empty = full + STAGES;
    uint64_t *done = empty + STAGES;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(done + 1);

    const int warp = threadIdx.x >> 5;
    const int tiles_w = g.w / g.bw, tiles_h = g.h / g.bh;
    int t = blockIdx.x;
    const int w0 = (t % tiles_w) * g.bw;
    t /= tiles_w;
    const int h0 = (t % tiles_h) * g.bh;
    const int img = t / tiles_h;
    const int n0 = blockIdx.y * g.bn;
    const uint32_t ncols = tmem_cols_for(g.bn);

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        fence_async_shared();
    }
    __syncwarp();
    if (warp == 0) tmem_alloc(tslot, ncols);
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    const uint32_t tmem = *tslot;

    const int nkc = g.cin / g.kc;
    const int nk = 9 * nkc;
    const uint32_t layout = umma_layout_for((int)aw);
    const uint32_t sbase = smem_u32(base);

    // warp 0 streams the operand boxes and warp 1 issues the MMAs; a whole warp runs
    // each loop (lane 0 waits and issues, the other lanes wait at the shuffle), so
    // no lane of a working warp spins on the accumulator barrier meanwhile
    const int lane = threadIdx.x & 31;
    if (warp == 0) {
        // producer: one A box (128 shifted pixels x kc channels) and one B box (bn x kc weights) per k-block
        for (int kb = 0; kb < nk; ++kb) {
            int fail = 0;
            if (lane == 0) {
                const int s = kb % STAGES;
                if (kb >= STAGES && !mbar_wait_bounded(&empty[s], ((kb / STAGES) - 1) & 1, NN_WAIT)) {
                    atomicExch(err, 1);
                    fail = 1;
                } else {
                    const int tap = kb / nkc, c0 = (kb % nkc) * g.kc;
                    mbar_arrive_expect_tx(&full[s], a_bytes + b_bytes);
                    tma_load_4d(base + s * st_bytes, &tmX, &full[s], c0, w0 + tap % 3 - 1, h0 + tap / 3 - 1, img);
                    tma_load_3d(base + s * st_bytes + a_bytes, &tmW, &full[s], c0, n0, tap);
                }
            }
            if (__shfl_sync(0xffffffffu, fail, 0)) break;
        }
    } else if (warp == 1) {
        // MMA issuer: kc/16 MMAs (K = 16) per k-block, the K step is +32 bytes inside the swizzle atom
        const uint32_t idesc = umma_idesc_bf16(128, g.bn, 0, 0);
        for (int kb = 0; kb < nk; ++kb) {
            int fail = 0;
            if (lane == 0) {
                const int s = kb % STAGES;
                if (!mbar_wait_bounded(&full[s], (kb / STAGES) & 1, NN_WAIT)) {
                    atomicExch(err, 2);
                    fail = 1;
                } else {
                    tmem_fence_after();
                    const uint32_t sa = sbase + s * st_bytes, sb = sa + a_bytes;
                    for (int k = 0; k < g.kc / 16; ++k) {
                        const uint64_t ad = umma_smem_desc(sa + 32u * k, 16u, 8u * aw, layout);
                        const uint64_t bd = umma_smem_desc(sb + 32u * k, 16u, 8u * aw, layout);
                        umma_bf16(tmem, ad, bd, idesc, (kb | k) != 0);
                    }
                    umma_commit(&empty[s]);
                }
            }
            if (__shfl_sync(0xffffffffu, fail, 0)) break;
        }
        if (lane == 0) umma_commit(done);
        __syncwarp();
    }

    // epilogue: thread m owns accumulator row m (TMEM lane m) = pixel m of the box
    const bool ok = mbar_wait_bounded(done, 0, NN_WAIT);
    if (!ok && (threadIdx.x & 31) == 0) atomicExch(err, 3);
    __syncwarp();
    tmem_fence_after();
    const int m = threadIdx.x;
    const size_t pix = ((size_t)img * g.h + h0 + m / g.bw) * g.w + w0 + m % g.bw;
    for (int c = 0; c < g.bn; c += 16) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
        const int ch = n0 + c;
        if (bias) {
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] += __ldg(bias + ch + i);
        }
        if (g.act == 1) {
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i], 0.f);
        }
        if (mask) {
            float mk[16];
            load_bf16x16(mask + pix * g.m_cstride + g.m_coff + ch, mk);
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = mk[i] > 0.f ? v[i] : 0.f;
        }
        if (ok) store_bf16x16(y + pix * g.y_cstride + g.y_coff + ch, v);
    }
    tmem_fence_before();
    __syncthreads();
    if (warp == 0) {
        tmem_fence_after();
        tmem_dealloc(tmem, ncols);
    }
}

// ------------------------------------------------------------------ weight gradient (MN-major)

__global__ void __launch_bounds__(CONV_THREADS, 1)
    k_conv_wgrad(const __grid_constant__ CUtensorMap tmDZ, const __grid_constant__ CUtensorMap tmX, WgradGeo g,
                 float *__restrict__ dw, int *err)
{
    const uint32_t aw_a = 2u * g.ae_a, aw_b = 2u * g.ae_b;
    const int na = 128 / g.ae_a, nb = g.bn / g.ae_b;       // atom columns along M and N
    const uint32_t col_a = WG_PIX * aw_a, col_b = WG_PIX * aw_b;  // bytes of one atom column (multiples of 1024)
    const uint32_t a_bytes = na * col_a, b_bytes = nb * col_b;
    const uint32_t st_bytes = a_bytes + b_bytes;
    uint8_t *base = align1024(nn_smem);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + STAGES * st_bytes);
    uint64_t *empty = full + STAGES;
    uint64_t *done = empty + STAGES;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(done + 1);

    const int warp = threadIdx.x >> 5;
    const int tap = blockIdx.z;
    const int m0 = (blockIdx.y / g.ci_tiles) * 128;
    const int n0 = (blockIdx.y % g.ci_tiles) * g.bn;
    const int c_begin = blockIdx.x * g.chunks_per_split;
    const int c_end = min(g.chunks, c_begin + g.chunks_per_split);
    const int nk = c_end - c_begin;
    const uint32_t ncols = tmem_cols_for(g.bn);
    int na_live = 0;                                        // atom columns of dz inside the channel range
    for (int a = 0; a < na; ++a) na_live += (m0 + a * g.ae_a < g.cout);

    // atom columns past the last output channel stay zero: clear them once in every stage
    for (int s = 0; s < STAGES; ++s) {
        uint32_t *p = reinterpret_cast<uint32_t *>(base + s * st_bytes + na_live * col_a);
        const int words = (na - na_live) * col_a / 4;
        for (int i = threadIdx.x; i < words; i += blockDim.x) p[i] = 0u;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
    }
    fence_async_shared();
    __syncwarp();
    if (warp == 0) tmem_alloc(tslot, ncols);
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t sbase = smem_u32(base);
    const int wchunks = g.w / WG_PIX;
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;

    const int lane = threadIdx.x & 31;
    if (warp == 0 && nk > 0) {
        for (int kb = 0; kb < nk; ++kb) {
            int fail = 0;
            if (lane == 0) {
                const int s = kb % STAGES;
                if (kb >= STAGES && !mbar_wait_bounded(&empty[s], ((kb / STAGES) - 1) & 1, NN_WAIT)) {
                    atomicExch(err, 11);
                    fail = 1;
                } else {
                    int c = c_begin + kb;
                    const int px0 = (c % wchunks) * WG_PIX;
                    c /= wchunks;
                    const int hh = c % g.h, img = c / g.h;
                    mbar_arrive_expect_tx(&full[s], na_live * col_a + b_bytes);
                    uint8_t *sa = base + s * st_bytes;
                    for (int a = 0; a < na_live; ++a)
                        tma_load_4d(sa + a * col_a, &tmDZ, &full[s], m0 + a * g.ae_a, px0, hh, img);
                    for (int b = 0; b < nb; ++b)
                        tma_load_4d(sa + a_bytes + b * col_b, &tmX, &full[s], n0 + b * g.ae_b, px0 + dx, hh + dy,
                                    img);
                }
            }
            if (__shfl_sync(0xffffffffu, fail, 0)) break;
        }
    } else if (warp == 1 && nk > 0) {
        // K = 16 pixel rows per MMA: +16 rows of the atom column; LBO = atom column stride, SBO = 8 rows
        const uint32_t idesc = umma_idesc_bf16(128, g.bn, 1, 1);
        const uint32_t la = umma_layout_for((int)aw_a), lb = umma_layout_for((int)aw_b);
        for (int kb = 0; kb < nk; ++kb) {
            int fail = 0;
            if (lane == 0) {
                const int s = kb % STAGES;
                if (!mbar_wait_bounded(&full[s], (kb / STAGES) & 1, NN_WAIT)) {
                    atomicExch(err, 12);
                    fail = 1;
                } else {
                    tmem_fence_after();
                    const uint32_t sa = sbase + s * st_bytes, sb = sa + a_bytes;
#pragma unroll
                    for (int k = 0; k < WG_PIX / 16; ++k) {
                        const uint64_t ad = umma_smem_desc(sa + 16u * aw_a * k, col_a, 8u * aw_a, la);
                        const uint64_t bd = umma_smem_desc(sb + 16u * aw_b * k, col_b, 8u * aw_b, lb);
                        umma_bf16(tmem, ad, bd, idesc, (kb | k) != 0);
                    }
                    umma_commit(&empty[s]);
                }
            }
            if (__shfl_sync(0xffffffffu, fail, 0)) break;
        }
        if (lane == 0) umma_commit(done);
        __syncwarp();
    }

    if (nk > 0) {
        const bool ok = mbar_wait_bounded(done, 0, NN_WAIT);
        if (!ok && (threadIdx.x & 31) == 0) atomicExch(err, 13);
        __syncwarp();
        tmem_fence_after();
        const int co = m0 + threadIdx.x;
        for (int c = 0; c < g.bn; c += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
            if (ok && co < g.cout) {
                float *dst = dw + ((size_t)tap * g.cout + co) * g.cin + n0 + c;
#pragma unroll
                for (int i = 0; i < 16; ++i) atomicAdd(dst + i, v[i]);
            }
        }
    }
    tmem_fence_before();
    __syncthreads();
    if (warp == 0) {
        tmem_fence_after();
        tmem_dealloc(tmem, ncols);
    }
}

// ------------------------------------------------------------------ plain kernels

// features [n][4][hd][wd] FP32 (channel scales applied) -> NHWC BF16 [n][h][w][16], zero outside
__global__ void k_pack_input(const float *__restrict__ f, int n, int hd, int wd, int h, int w, float s0, float s1,
                             float s2, float s3, __nv_bfloat16 *__restrict__ x)
{
    const size_t total = (size_t)n * h * w;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(p % w), i = (int)((p / w) % h), img = (int)(p / ((size_t)w * h));
        float v[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = 0.f;
        if (i < hd && j < wd) {
            const size_t plane = (size_t)hd * wd, o = (size_t)img * 4 * plane + (size_t)i * wd + j;
            v[0] = f[o] * s0;
            v[1] = f[o + plane] * s1;
            v[2] = f[o + 2 * plane] * s2;
            v[3] = f[o + 3 * plane] * s3;
        }
        store_bf16x16(x + p * 16, v);
    }
}

// 2x2 average pool of a channel slice: in [n][h][w][in_cstride] at in_coff -> out [n][h/2][w/2][c]
__global__ void k_avgpool2(const __nv_bfloat16 *__restrict__ in, int n, int h, int w, int c, int in_cstride,
                           int in_coff, __nv_bfloat16 *__restrict__ out)
{
    const int ho = h / 2, wo = w / 2;
    const size_t total = (size_t)n * ho * wo * c;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int ch = (int)(e % c);
        size_t p = e / c;
        const int j = (int)(p % wo), i = (int)((p / wo) % ho), img = (int)(p / ((size_t)wo * ho));
        const size_t r0 = ((size_t)img * h + 2 * i) * w + 2 * j;
        const __nv_bfloat16 *q = in + in_coff + ch;
        const float s = __bfloat162float(q[r0 * in_cstride]) + __bfloat162float(q[(r0 + 1) * in_cstride]) +
                        __bfloat162float(q[(r0 + w) * in_cstride]) + __bfloat162float(q[(r0 + w + 1) * in_cstride]);
        out[e] = __float2bfloat16_rn(0.25f * s);
    }
}

// gradient of a skip tensor y (a ReLU output stored in a concatenation buffer slice):
// dz = (dcat[slice] + 1/4 dpool[parent]) * [y > 0]  -> contiguous [n][h][w][c]
__global__ void k_skip_grad(const __nv_bfloat16 *__restrict__ dcat, const __nv_bfloat16 *__restrict__ ycat,
                            int cstride, int coff, const __nv_bfloat16 *__restrict__ dpool, int n, int h, int w, int c,
                            __nv_bfloat16 *__restrict__ dz)
{
    const size_t total = (size_t)n * h * w * c;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int ch = (int)(e % c);
        const size_t p = e / c;
        const int j = (int)(p % w), i = (int)((p / w) % h), img = (int)(p / ((size_t)w * h));
        const size_t pp = ((size_t)img * (h / 2) + i / 2) * (w / 2) + j / 2;
        float v = 0.25f * __bfloat162float(dpool[pp * c + ch]);
        if (dcat) v += __bfloat162float(dcat[p * cstride + coff + ch]);
        dz[e] = __float2bfloat16_rn(__bfloat162float(ycat[p * cstride + coff + ch]) > 0.f ? v : 0.f);
    }
}

// nearest 2x upsampling of low [n][h][w][c] into channels [0, c) of out [n][2h][2w][out_cstride]
__global__ void k_upsample2(const __nv_bfloat16 *__restrict__ low, int n, int h, int w, int c, int out_cstride,
                            __nv_bfloat16 *__restrict__ out)
{
    const int ho = 2 * h, wo = 2 * w;
    const size_t total = (size_t)n * ho * wo * c;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int ch = (int)(e % c);
        const size_t p = e / c;
        const int j = (int)(p % wo), i = (int)((p / wo) % ho), img = (int)(p / ((size_t)wo * ho));
        out[p * out_cstride + ch] = low[(((size_t)img * h + i / 2) * w + j / 2) * c + ch];
    }
}

// gradient through the upsampling into a ReLU output: dz[low] = sum_{2x2} dcat[.., 0:c] * [low > 0]
__global__ void k_upsample2_grad(const __nv_bfloat16 *__restrict__ dcat, int cstride,
                                 const __nv_bfloat16 *__restrict__ low, int n, int h, int w, int c,
                                 __nv_bfloat16 *__restrict__ dz)
{
    const size_t total = (size_t)n * h * w * c;
    const int wo = 2 * w;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int ch = (int)(e % c);
        const size_t p = e / c;
        const int j = (int)(p % w), i = (int)((p / w) % h), img = (int)(p / ((size_t)w * h));
        const size_t r0 = ((size_t)img * 2 * h + 2 * i) * wo + 2 * j;
        const float s = __bfloat162float(dcat[r0 * cstride + ch]) + __bfloat162float(dcat[(r0 + 1) * cstride + ch]) +
                        __bfloat162float(dcat[(r0 + wo) * cstride + ch]) +
                        __bfloat162float(dcat[(r0 + wo + 1) * cstride + ch]);
        dz[e] = __float2bfloat16_rn(__bfloat162float(low[e]) > 0.f ? s : 0.f);
    }
}

// 1x1 output head: out[p] = b + sum_c wt[c] y[p][c], y [npix][c] BF16 (c <= 64)
__global__ void k_head_fwd(const __nv_bfloat16 *__restrict__ y, size_t npix, int c, const float *__restrict__ wt,
                           const float *__restrict__ b, float *__restrict__ out)
{
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < npix; p += (size_t)gridDim.x * blockDim.x) {
        float s = b[0];
        for (int k = 0; k < c; k += 16) {
            float v[16];
            load_bf16x16(y + p * c + k, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) s = fmaf(__ldg(wt + k + i), v[i], s);
        }
        out[p] = s;
    }
}

// masked mean-square loss of the head and its gradient:
// L = sum_p wgt[p] (out - target)^2 / norm;  dz[p][c] = dL/dout * wt[c] * [y > 0];
// dwt[c] += sum_p dL/dout y[p][c];  db += sum_p dL/dout;  loss (FP64) += L
__global__ void k_head_loss_grad(const __nv_bfloat16 *__restrict__ y, size_t npix, int c,
                                 const float *__restrict__ wt, const float *__restrict__ out,
                                 const float *__restrict__ target, const float *__restrict__ wgt, float inv_norm,
                                 __nv_bfloat16 *__restrict__ dz, float *__restrict__ dwt, float *__restrict__ db,
                                 double *__restrict__ loss)
{
    __shared__ float s_dw[64];
    __shared__ float s_db;
    __shared__ double s_l;
    for (int i = threadIdx.x; i < 64; i += blockDim.x) s_dw[i] = 0.f;
    if (threadIdx.x == 0) {
        s_db = 0.f;
        s_l = 0.0;
    }
    __syncthreads();
    float acc_db = 0.f;
    double acc_l = 0.0;
    float acc_dw[64];
    for (int i = 0; i < 64; ++i) acc_dw[i] = 0.f;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < npix; p += (size_t)gridDim.x * blockDim.x) {
        const float r = out[p] - target[p];
        const float wp = wgt[p];
        acc_l += (double)wp * r * r * inv_norm;
        const float g = 2.f * wp * r * inv_norm;
        acc_db += g;
        for (int k = 0; k < c; k += 16) {
            float v[16], d[16];
            load_bf16x16(y + p * c + k, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                acc_dw[k + i] = fmaf(g, v[i], acc_dw[k + i]);
                d[i] = v[i] > 0.f ? g * __ldg(wt + k + i) : 0.f;
            }
            store_bf16x16(dz + p * c + k, d);
        }
    }
    for (int i = 0; i < c; ++i) atomicAdd(&s_dw[i], acc_dw[i]);
    atomicAdd(&s_db, acc_db);
    atomicAdd(&s_l, acc_l);
    __syncthreads();
    if (threadIdx.x < c) atomicAdd(dwt + threadIdx.x, s_dw[threadIdx.x]);
    if (threadIdx.x == 0) {
        atomicAdd(db, s_db);
        atomicAdd(loss, s_l);
    }
}

// db[c] += sum over pixels of dz[p][c] (NHWC contiguous, c <= 1024)
__global__ void k_bias_grad(const __nv_bfloat16 *__restrict__ dz, size_t npix, int c, float *__restrict__ db)
{
    extern __shared__ float s_b[];
    for (int i = threadIdx.x; i < c; i += blockDim.x) s_b[i] = 0.f;
    __syncthreads();
    const size_t total = npix * c;
    // the stride is a multiple of c, so each thread stays on one channel
    const size_t stride = (size_t)gridDim.x * blockDim.x / c * c;
    const size_t start = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (stride > 0 && start < stride) {
        float s = 0.f;
        for (size_t e = start; e < total; e += stride) s += __bfloat162float(dz[e]);
        atomicAdd(&s_b[start % c], s);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < c; i += blockDim.x) atomicAdd(db + i, s_b[i]);
}

// FP32 master weights [9][cout][cin] -> BF16 forward layout (same) and input-gradient
// layout wt_t[8 - tap][cin][cout] (taps flipped, channels transposed)
__global__ void k_pack_weights(const float *__restrict__ w32, int cout, int cin, __nv_bfloat16 *__restrict__ wf,
                               __nv_bfloat16 *__restrict__ wt)
{
    const int total = 9 * cout * cin;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int ci = e % cin, co = (e / cin) % cout, tap = e / (cin * cout);
        const __nv_bfloat16 v = __float2bfloat16_rn(w32[e]);
        wf[e] = v;
        if (wt) wt[((size_t)(8 - tap) * cin + ci) * cout + co] = v;
    }
}

// Adam in the efficient form of Kingma and Ba (bias corrections folded into
// lr_t by the host, eps added to sqrt(v)); gradients cleared afterwards
__global__ void k_adam(float *__restrict__ p, float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       size_t n, float lr_t, float b1, float b2, float eps, float grad_scale)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i] * grad_scale;
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr_t * mi / (sqrtf(vi) + eps);
        g[i] = 0.f;
    }
}

}  // namespace nn
}  // namespace stfwi

// ================================================================== C ABI

using namespace stfwi;
using namespace stfwi::nn;

namespace {

thread_local std::string g_err;

int nn_fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

PFN_cuTensorMapEncodeTiled_v12000 nn_encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

CUtensorMapSwizzle swizzle_for(int atom_bytes)
{
    return atom_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                             : atom_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
}

// BF16 tensor of `rank` dims (dims[0] contiguous), box `box`, swizzle matching box[0] * 2 bytes
int encode_bf16(CUtensorMap *m, const void *base, int rank, const cuuint64_t *dims, const cuuint32_t *box)
{
    auto fn = nn_encode_fn();
    if (!fn) return nn_fail(STFWI_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    cuuint64_t strides[4];
    cuuint64_t s = dims[0] * 2;
    for (int i = 1; i < rank; ++i) {
        strides[i - 1] = s;
        s *= dims[i];
    }
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, rank, const_cast<void *>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for((int)box[0] * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return nn_fail(STFWI_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return STFWI_OK;
}

int check_launch(const char *what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return nn_fail(STFWI_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return STFWI_OK;
}

constexpr int NN_MAX_DEVICES = 64;

// one pipeline error flag per device (a kernel writes the flag of its own device)
// the status word of the pipeline waits: a device variable of this module,
// zero when the module loads on a device; its address is looked up once per
// device (under a lock), so no network op allocates or synchronises for it
__device__ int g_nn_err_flag;

int *err_flag()
{
    static std::mutex mu;
    static int *flags[NN_MAX_DEVICES] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NN_MAX_DEVICES) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!flags[dev]) {
        int *f = nullptr;
        if (cudaGetSymbolAddress((void **)&f, g_nn_err_flag) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        flags[dev] = f;
    }
    return flags[dev];
}

// the dynamic shared-memory limit of a kernel is set once per device
template <typename K>
int smem_limit_once(K kern, size_t bytes, bool (&done)[NN_MAX_DEVICES], const char *what)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NN_MAX_DEVICES)
        return nn_fail(STFWI_ERR_CUDA, "%s: no usable current device", what);
    if (!done[dev]) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
            return check_launch(what);
        done[dev] = true;
    }
    return STFWI_OK;
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int largest_atom(int c) { return c % 64 == 0 ? 64 : c % 32 == 0 ? 32 : 16; }

// Shared memory per SM is 228 KB (1 KB of it reserved per block); a launch asks for at
// least 228 KB / (512 / tensor-memory columns) so that the CTAs resident on one SM never
// hold more than the SM's 512 tensor-memory columns and tcgen05.alloc never waits.
size_t tmem_floor(int bn)
{
    const size_t per_sm = 233472, ctas = 512 / tmem_cols_for(bn);
    return per_sm / ctas - 1024 + 16;
}

size_t conv_smem(int kc, int bn)
{
    const size_t aw = 2 * kc, a = 128 * aw, b = ((size_t)bn * aw + 1023) & ~(size_t)1023;
    const size_t need = 1024 + STAGES * (a + b) + (2 * STAGES + 1) * 8 + 16;
    return need > tmem_floor(bn) ? need : tmem_floor(bn);
}

size_t wgrad_smem(int bn)
{
    const size_t need = 1024 + STAGES * (size_t)(128 + bn) * WG_PIX * 2 + (2 * STAGES + 1) * 8 + 16;
    return need > tmem_floor(bn) ? need : tmem_floor(bn);
}

int conv_common(const void *x, int n, int h, int w, int cin, const void *wt, int cout, const float *bias, int act,
                const void *mask, int m_cstride, int m_coff, void *y, int y_cstride, int y_coff, cudaStream_t st)
{
    if (n <= 0 || h <= 0 || w <= 0) return nn_fail(STFWI_ERR_INVALID, "conv: empty image batch");
    if (cin % 16 || cout % 16 || cin <= 0 || cout <= 0)
        return nn_fail(STFWI_ERR_INVALID, "conv: channel counts must be positive multiples of 16 (%d, %d)", cin, cout);
    const int bw = w >= 128 ? 128 : w;
    if (w % bw || 128 % bw || h % (128 / bw))
        return nn_fail(STFWI_ERR_INVALID, "conv: %dx%d does not tile into 128-pixel boxes", h, w);
    if (y_cstride % 8 || y_coff % 8 || y_coff + cout > y_cstride)
        return nn_fail(STFWI_ERR_INVALID, "conv: output channel stride/offset must be multiples of 8 and hold cout");
    if (mask && (m_cstride % 8 || m_coff % 8 || m_coff + cout > m_cstride))
        return nn_fail(STFWI_ERR_INVALID, "conv: mask channel stride/offset");
    if (!aligned16(x) || !aligned16(wt) || !aligned16(y) || (mask && !aligned16(mask)))
        return nn_fail(STFWI_ERR_INVALID, "conv: tensors must be 16-byte aligned");
    ConvGeo g{};
    g.n = n; g.h = h; g.w = w; g.cin = cin; g.cout = cout;
    g.kc = largest_atom(cin);
    g.bn = cout % 128 == 0 ? 128 : cout % 64 == 0 ? 64 : cout % 32 == 0 ? 32 : 16;
    g.bw = bw; g.bh = 128 / bw;
    g.y_cstride = y_cstride; g.y_coff = y_coff; g.act = act;
    g.m_cstride = m_cstride; g.m_coff = m_coff;
    CUtensorMap tx, tw;
    const cuuint64_t dx[4] = {(cuuint64_t)cin, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
    const cuuint32_t bx[4] = {(cuuint32_t)g.kc, (cuuint32_t)g.bw, (cuuint32_t)g.bh, 1};
    int rc = encode_bf16(&tx, x, 4, dx, bx);
    if (rc) return rc;
    const cuuint64_t dw[3] = {(cuuint64_t)cin, (cuuint64_t)cout, 9};
    const cuuint32_t bwx[3] = {(cuuint32_t)g.kc, (cuuint32_t)g.bn, 1};
    rc = encode_bf16(&tw, wt, 3, dw, bwx);
    if (rc) return rc;
    int *err = err_flag();
    if (!err) return nn_fail(STFWI_ERR_CUDA, "conv: the error flag of this device could not be looked up");
    static bool attr[NN_MAX_DEVICES] = {};
    rc = smem_limit_once(k_conv_kmajor, conv_smem(64, 128), attr, "conv: shared-memory attribute");
    if (rc) return rc;
    const dim3 grid((unsigned)((size_t)n * (h / g.bh) * (w / g.bw)), (unsigned)(cout / g.bn));
    k_conv_kmajor<<<grid, CONV_THREADS, conv_smem(g.kc, g.bn), st>>>(
        tx, tw, g, bias, static_cast<const __nv_bfloat16 *>(mask), static_cast<__nv_bfloat16 *>(y), err);
    return check_launch("k_conv_kmajor");
}

unsigned blocks_for(size_t n, int threads)
{
    size_t b = (n + threads - 1) / threads;
    return (unsigned)(b < 1 ? 1 : b > 4 * 148 * 8 ? 4 * 148 * 8 : b);
}

}  // namespace

extern "C" {

const char *stfwi_nn_last_error(void) { return g_err.c_str(); }

int stfwi_nn_check(void *stream)
{
    int *err = err_flag();
    if (!err) return nn_fail(STFWI_ERR_CUDA, "the error flag of this device could not be looked up");
    int v = 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(&v, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return check_launch("stfwi_nn_check");
    if (v) {
        cudaMemsetAsync(err, 0, sizeof(int), st);
        cudaStreamSynchronize(st);
        return nn_fail(STFWI_ERR_CUDA, "a tensor-core pipeline wait gave up (code %d)", v);
    }
    return STFWI_OK;
}

int stfwi_nn_conv3x3(const void *x, int n, int h, int w, int cin, const void *wt, int cout, const float *bias,
                     int relu, void *y, int y_cstride, int y_coff, void *stream)
{
    return conv_common(x, n, h, w, cin, wt, cout, bias, relu ? 1 : 0, nullptr, 0, 0, y, y_cstride, y_coff,
                       static_cast<cudaStream_t>(stream));
}

int stfwi_nn_conv3x3_dgrad(const void *dz, int n, int h, int w, int cout, const void *wt_t, int cin,
                           const void *mask, int m_cstride, int m_coff, void *dx, void *stream)
{
    return conv_common(dz, n, h, w, cout, wt_t, cin, nullptr, 0, mask, m_cstride, m_coff, dx, cin, 0,
                       static_cast<cudaStream_t>(stream));
}

int stfwi_nn_conv3x3_wgrad(const void *x, const void *dz, int n, int h, int w, int cin, int cout, float *dw,
                           void *stream)
{
    if (n <= 0 || h <= 0 || w <= 0) return nn_fail(STFWI_ERR_INVALID, "wgrad: empty image batch");
    if (cin % 16 || cout % 16 || cin <= 0 || cout <= 0)
        return nn_fail(STFWI_ERR_INVALID, "wgrad: channel counts must be positive multiples of 16");
    if (w % WG_PIX) return nn_fail(STFWI_ERR_INVALID, "wgrad: width must be a multiple of %d", WG_PIX);
    if (!aligned16(x) || !aligned16(dz) || !aligned16(dw))
        return nn_fail(STFWI_ERR_INVALID, "wgrad: tensors must be 16-byte aligned");
    WgradGeo g{};
    g.n = n; g.h = h; g.w = w; g.cout = cout; g.cin = cin;
    g.ae_a = largest_atom(cout);
    g.bn = cin % 128 == 0 ? 128 : cin % 64 == 0 ? 64 : cin % 32 == 0 ? 32 : 16;
    g.ae_b = g.bn >= 64 ? 64 : g.bn;
    g.ci_tiles = cin / g.bn;
    const int co_tiles = (cout + 127) / 128;
    g.chunks = n * h * (w / WG_PIX);
    const int tiles = 9 * co_tiles * g.ci_tiles;
    int splits = (4 * 148 + tiles - 1) / tiles;
    if (splits > g.chunks) splits = g.chunks;
    if (splits < 1) splits = 1;
    g.chunks_per_split = (g.chunks + splits - 1) / splits;
    splits = (g.chunks + g.chunks_per_split - 1) / g.chunks_per_split;
    CUtensorMap ta, tb;
    const cuuint64_t da[4] = {(cuuint64_t)cout, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
    const cuuint32_t ba[4] = {(cuuint32_t)g.ae_a, WG_PIX, 1, 1};
    int rc = encode_bf16(&ta, dz, 4, da, ba);
    if (rc) return rc;
    const cuuint64_t db[4] = {(cuuint64_t)cin, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
    const cuuint32_t bb[4] = {(cuuint32_t)g.ae_b, WG_PIX, 1, 1};
    rc = encode_bf16(&tb, x, 4, db, bb);
    if (rc) return rc;
    int *err = err_flag();
    if (!err) return nn_fail(STFWI_ERR_CUDA, "wgrad: the error flag of this device could not be looked up");
    static bool attr[NN_MAX_DEVICES] = {};
    rc = smem_limit_once(k_conv_wgrad, wgrad_smem(128), attr, "wgrad: shared-memory attribute");
    if (rc) return rc;
    const dim3 grid((unsigned)splits, (unsigned)(co_tiles * g.ci_tiles), 9);
    k_conv_wgrad<<<grid, CONV_THREADS, wgrad_smem(g.bn), static_cast<cudaStream_t>(stream)>>>(ta, tb, g, dw, err);
    return check_launch("k_conv_wgrad");
}

int stfwi_nn_pack_input(const float *feat, int n, int hd, int wd, int h, int w, const float *scale4, void *x,
                        void *stream)
{
    if (hd > h || wd > w || n <= 0) return nn_fail(STFWI_ERR_INVALID, "pack_input: sizes");
    const size_t total = (size_t)n * h * w;
    k_pack_input<<<blocks_for(total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        feat, n, hd, wd, h, w, scale4[0], scale4[1], scale4[2], scale4[3], static_cast<__nv_bfloat16 *>(x));
    return check_launch("k_pack_input");
}

int stfwi_nn_avgpool2(const void *in, int n, int h, int w, int c, int in_cstride, int in_coff, void *out,
                      void *stream)
{
    if (h % 2 || w % 2) return nn_fail(STFWI_ERR_INVALID, "avgpool2: odd size");
    const size_t total = (size_t)n * (h / 2) * (w / 2) * c;
    k_avgpool2<<<blocks_for(total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16 *>(in), n, h, w, c, in_cstride, in_coff, static_cast<__nv_bfloat16 *>(out));
    return check_launch("k_avgpool2");
}

int stfwi_nn_skip_grad(const void *dcat, const void *ycat, int cstride, int coff, const void *dpool, int n, int h,
                       int w, int c, void *dz, void *stream)
{
    const size_t total = (size_t)n * h * w * c;
    k_skip_grad<<<blocks_for(total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16 *>(dcat), static_cast<const __nv_bfloat16 *>(ycat), cstride, coff,
        static_cast<const __nv_bfloat16 *>(dpool), n, h, w, c, static_cast<__nv_bfloat16 *>(dz));
    return check_launch("k_skip_grad");
}

int stfwi_nn_upsample2(const void *low, int n, int h, int w, int c, int out_cstride, void *out, void *stream)
{
    const size_t total = (size_t)n * 4 * h * w * c;
    k_upsample2<<<blocks_for(total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16 *>(low), n, h, w, c, out_cstride, static_cast<__nv_bfloat16 *>(out));
    return check_launch("k_upsample2");
}

int stfwi_nn_upsample2_grad(const void *dcat, int cstride, const void *low, int n, int h, int w, int c, void *dz,
                            void *stream)
{
    const size_t total = (size_t)n * h * w * c;
    k_upsample2_grad<<<blocks_for(total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16 *>(dcat), cstride, static_cast<const __nv_bfloat16 *>(low), n, h, w, c,
        static_cast<__nv_bfloat16 *>(dz));
    return check_launch("k_upsample2_grad");
}

int stfwi_nn_head(const void *y, size_t npix, int c, const float *wt, const float *b, float *out, void *stream)
{
    if (c % 16 || c > 64) return nn_fail(STFWI_ERR_INVALID, "head: channels must be a multiple of 16, <= 64");
    k_head_fwd<<<blocks_for(npix, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16 *>(y), npix, c, wt, b, out);
    return check_launch("k_head_fwd");
}

int stfwi_nn_head_loss_grad(const void *y, size_t npix, int c, const float *wt, const float *out,
                            const float *target, const float *wgt, float inv_norm, void *dz, float *dwt, float *db,
                            double *loss, void *stream)
{
    if (c % 16 || c > 64) return nn_fail(STFWI_ERR_INVALID, "head: channels must be a multiple of 16, <= 64");
    unsigned blocks = blocks_for(npix, 256);
    if (blocks > 1184) blocks = 1184;
    k_head_loss_grad<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16 *>(y), npix, c, wt, out, target, wgt, inv_norm,
        static_cast<__nv_bfloat16 *>(dz), dwt, db, loss);
    return check_launch("k_head_loss_grad");
}

int stfwi_nn_bias_grad(const void *dz, size_t npix, int c, float *db, void *stream)
{
    if (c <= 0 || c > 1024) return nn_fail(STFWI_ERR_INVALID, "bias_grad: channel count %d", c);
    const int threads = 256;
    unsigned blocks = blocks_for(npix * c / 64, threads);
    if (blocks * threads < (unsigned)c) blocks = (c + threads - 1) / threads;
    k_bias_grad<<<blocks, threads, c * sizeof(float), static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16 *>(dz), npix, c, db);
    return check_launch("k_bias_grad");
}

int stfwi_nn_pack_weights(const float *w32, int cout, int cin, void *wf, void *wt, void *stream)
{
    const int total = 9 * cout * cin;
    k_pack_weights<<<blocks_for(total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        w32, cout, cin, static_cast<__nv_bfloat16 *>(wf), static_cast<__nv_bfloat16 *>(wt));
    return check_launch("k_pack_weights");
}

int stfwi_nn_adam(float *p, float *g, float *m, float *v, size_t n, float lr_t, float b1, float b2, float eps,
                  float grad_scale, void *stream)
{
    k_adam<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(p, g, m, v, n, lr_t, b1, b2, eps,
                                                                            grad_scale);
    return check_launch("k_adam");
}

}  // extern "C"
