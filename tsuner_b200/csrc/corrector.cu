// corrector.cu -- learned corrector: a 6-layer, 32-channel 3x3 convolutional
// network that lifts coarse-grid maximum-depth / bed-change maps to the fine
// grid.  Its convolutions (forward, input gradient, weight gradient) run on
// the 5th-generation tensor cores (tcgen05.mma, BF16 operands from shared
// memory, FP32 accumulators in TMEM); the rest of the training loop
// (feature assembly, loss, Adam) is small elementwise kernels.
// No counterpart in the reference.
//
// Tensors: activations NHWC BF16 with 32 channels ([img][y][x][32]);
// weights BF16 Wk[cout][tap][cin], tap = (dy+1)*3 + (dx+1) (so that
// Y[y][x] = sum W[tap] X[y+dy][x+dx], zero padding); FP32 master weights,
// bias and Adam moments.
//
// Forward / input-gradient convolution (conv3x3_fwd_kernel): implicit GEMM
//   D[128 pixels x 32 cout] = sum over 9 taps x 2 channel halves of
//   A_tap,h[128 x 16] . B_tap,h[16 x 32]  (18 MMAs of M=128, N=32, K=16)
// over an 8 x 16 pixel tile.  The input patch (10 x 18 pixels with the halo)
// is stored in shared memory as four channel-quarter planes (16 bytes per
// pixel per plane), which makes every A_tap,h a K-major no-swizzle operand
// that starts inside the patch: core matrix = 8 consecutive pixels of one
// tile row (16-byte rows), the two K chunks one plane apart (LBO = plane
// size) and the 16 row groups one patch row apart (SBO = 160 B).  No im2col
// copy is made.  The patch arrives by TMA: four 4-D box loads per tile (one
// per channel quarter, zero fill outside the image = the convolution's
// padding) completing on an mbarrier.  CTAs are persistent; the patch and the
// TMEM accumulator are double-buffered so that the load of tile i+1 and the
// epilogue of tile i-1 overlap the MMAs of tile i.
//
// Weight gradient (conv3x3_wgrad_kernel): dW[cout][tap][cin] =
//   sum_p dZ[p][cout] X[p + off(tap)][cin], a GEMM with the pixels as the
// reduction dimension.  The input patch is loaded by one TMA box of a 5-D
// view of the NHWC tensor that lands as [row][channel quarter][x][8
// channels]: for a horizontal tap offset dx, the 12 core-matrix groups
// (dy, quarter) of the shifted patch are then 160 B apart, so
// D_dx[dy * 32 + cin][cout] is one M = 128 MMA per 16 pixels with A read in
// place (rows 96..127 see the next patch row and are ignored) and B = the dZ
// tile as loaded; no operand copy is made.  Three accumulators (dx = 0..2)
// take 96 TMEM columns.  Two stages: the next tile loads while this one's
// MMAs run.  The bias gradient is summed from the dZ tile on the CUDA cores.
// Each CTA accumulates a strip of tiles in TMEM and adds its partial result
// to the FP32 gradients with atomics.
//
// Every mbarrier wait is bounded (globaltimer); on expiry the kernel sets
// the error word, waits once more (bounded) for its MMAs, frees its TMEM and
// returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "hostio.h"
#include "async.cuh"
#include "tsuner_b200.h"

namespace tsu {
namespace corr {

typedef __nv_bfloat16 bf16;

constexpr int C = 32;                       // channels
constexpr int TXP = 8, TYP = 16;            // output tile (128 pixels)
constexpr int PW = TXP + 2, PH = TYP + 2;   // patch 10 x 18
constexpr int PPIX = PW * PH;               // 180
constexpr int kPlaneData = PPIX * 16;       // one channel-quarter plane: 2880 B
constexpr int kPlane = 2944;                // plane stride: 23 x 128 B (TMA destinations 128-byte aligned)
constexpr int kPatch = 4 * kPlane;          // 11776 B
constexpr int kWBytes = 9 * 4 * 32 * 16;    // weights: 18432 B
constexpr int KROWS = 9 * C;                // 288

// patch buffers: tile i+1 loads while tile i's MMAs run and tile i-1's
// epilogue stages its output in the buffer tile i-1 was read from
constexpr int kFwdBufs = 3;
constexpr int kFwdSmem = 1024 + kWBytes + kFwdBufs * kPatch + 64;
constexpr int kFwdCtasPerSm = 4;  // 4 x (54 KB + 1 KB) of shared memory, 4 x 64 TMEM columns
static_assert(kFwdCtasPerSm * (kFwdSmem + 1024) <= 228 * 1024 && kFwdCtasPerSm * 64 <= 512, "fwd residency");
static_assert(kPlane % 128 == 0 && kPlane >= kPlaneData && kWBytes % 128 == 0, "TMA destinations");
// warp-specialised forward (conv3x3_fwd_ws_kernel): warp 0 loads patches,
// warp 1 issues the MMAs, warps 2-5 run the epilogue.  A ring of kWsBufs
// patch buffers (full / empty barriers) and kWsAcc TMEM accumulators of 32
// columns (full / empty barriers); the epilogue stages its output in a 2 KB
// area per warp of its own.
constexpr int kWsBufs = 6, kWsAcc = 4, kWsThreads = 192;
constexpr int kWsStage = 4 * 2048;
constexpr int kWsBarBytes = (2 * kWsBufs + 2 * kWsAcc) * 8 + 32;
constexpr int kWsSmem = 1024 + kWBytes + kWsBufs * kPatch + kWsStage + kWsBarBytes;
constexpr int kWsCtasPerSm = 2;  // 2 x (~98 KB + 1 KB) of shared memory, 2 x 128 TMEM columns
static_assert(kWsCtasPerSm * (kWsSmem + 1024) <= 228 * 1024 && kWsCtasPerSm * 32 * kWsAcc <= 512, "ws residency");
// wgrad: patch + dZ tile + A for half of the 8 K steps (4 x 3 M blocks x 4 KB);
// ~67 KB, so three CTAs fit on an SM
constexpr int kZPlane = 128 * 16;
// weight gradient: the patch as [row][channel quarter][x][8 channels]
constexpr int kRowQ = 4 * PW * 16;           // one patch row: 640 B
constexpr int kWgPatch = PH * kRowQ;         // 11520 B
constexpr int kWgPatchBuf = 12288;           // + the row read by the ignored A rows 96..127
constexpr int kWgStage = kWgPatchBuf + 4 * kZPlane;
constexpr int kWgSmem = 1024 + 2 * kWgStage + 64;
constexpr int kWgCtasPerSm = 4;              // 128 TMEM columns each
static_assert(kWgPatch + kRowQ <= kWgPatchBuf && kWgPatchBuf % 128 == 0 && kWgStage % 128 == 0, "wgrad buffers");
static_assert(kWgCtasPerSm * (kWgSmem + 1024) <= 228 * 1024 && kWgCtasPerSm * 128 <= 512, "wgrad residency");

__device__ int g_corr_err;  // set by a kernel whose wait expired

// UMMA shared-memory descriptor, no swizzle, sm100 version field
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// kind::f16 instruction descriptor: D FP32, A/B BF16, majors, N, M
__host__ __device__ constexpr uint32_t idesc(int M, int N, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t id, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(id), "r"(accum)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// thread `lane` of the warp receives TMEM lane (base + lane), 32 columns
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}

struct TileGeom {
    int ntx, nty, per_img, total;
};
__host__ __device__ inline TileGeom tile_geom(int nimg, int H, int W) {
    TileGeom g;
    g.ntx = (W + TXP - 1) / TXP;
    g.nty = (H + TYP - 1) / TYP;
    g.per_img = g.ntx * g.nty;
    g.total = nimg * g.per_img;
    return g;
}

// 10 x 18 x 32 input patch (zero fill outside the image) -> four
// channel-quarter planes: one TMA box (8 channels x 10 x 18) per plane.  The
// innermost coordinate (channel 8q) is a multiple of 16 bytes; the halo may
// start at x0 - 1 = -1 or y0 - 1 = -1, which loads zeros.
__device__ __forceinline__ void issue_patch(const CUtensorMap *map, int img, int x0, int y0, unsigned char *patch,
                                            uint64_t *bar) {
#pragma unroll
    for (int q = 0; q < 4; q++) tma_load_4d(patch + q * kPlane, map, 8 * q, x0 - 1, y0 - 1, img, bar);
}

struct ConvArgs {
    const bf16 *X;
    int nimg, H, W;
    const bf16 *Wk;      // [cout][tap][cin]
    const float *bias;   // [32] or null
    int relu;            // apply max(., 0)
    const bf16 *gate;    // optional: zero output channel n where gate[p][n] <= 0
    bf16 *Ybf;           // BF16 output, or
    float *Yf;           // FP32 output, or
    float *Y2;           // FP32 output of channels 0 and 1 only, [pixel][2] (the corrector's last layer)
};

// Epilogue of one tile: TMEM accumulators (lane = pixel, column = output
// channel) + bias, ReLU, optional gate, then the store.  A warp holds 32
// pixels = 4 tile rows of 8; in NHWC each tile row is one contiguous run of
// 8 x 32 channels.  BF16 output (every layer but the last, and the input
// gradients) goes through `stage` (2 KB per warp, the patch buffer the tile's
// MMAs have finished reading): each lane writes its pixel's 4 x 16 B, then
// each instruction stores one tile row as 32 lanes x 16 B contiguous.
// 16-byte chunk k of pixel p sits in slot p * 4 + (k ^ ((p >> 1) & 3)), so
// both patterns are free of bank conflicts.  FP32 output (the last layer)
// goes the same way in two halves of 16 channels.  The gate is read per
// pixel (staging it too measured slower: 131 vs 110 us per 8 x 512^2 launch).
__device__ __forceinline__ void conv_epilogue(const ConvArgs &a, const TileGeom &G, int t, uint32_t taddr, int warp,
                                              int lane, const float *sBias, unsigned char *stage,
                                              uint64_t *release = nullptr) {
    const int img = t / G.per_img, r = t - img * G.per_img;
    const int tyi = r / G.ntx, txi = r - tyi * G.ntx;
    const int x0 = txi * TXP, y0 = tyi * TYP;
    // this lane's pixel (TMEM lane = pixel: 8 per tile row, 4 rows per warp)
    const int gx = x0 + (lane & 7), gy = y0 + warp * 4 + (lane >> 3);
    const bool inside = gx < a.W && gy < a.H;
    const long long o = inside ? (((long long)img * a.H + gy) * a.W + gx) * C : 0;
    // the gate (4 x 16 B of this pixel; the lines stay in L1 across the 4
    // loads) is requested before the TMEM read so the two latencies overlap
    uint4 g[4];
    if (a.gate && inside) {
        const uint4 *gp = reinterpret_cast<const uint4 *>(a.gate + o);
#pragma unroll
        for (int k = 0; k < 4; k++) g[k] = __ldg(gp + k);
    }
    float acc[32];
    tmem_ld32(taddr + ((uint32_t)(warp * 32) << 16), acc);
    if (release) {  // the accumulator is in registers: hand its TMEM columns back to the MMA issuer
        fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(release);
    }
#pragma unroll
    for (int n = 0; n < 32; n++) {
        float v = acc[n] + sBias[n];
        if (a.relu) v = fmaxf(v, 0.f);
        acc[n] = v;
    }
    if (a.gate && inside) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint32_t w[4] = {g[k].x, g[k].y, g[k].z, g[k].w};
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162 *>(&w[j]);
                if (!(__low2float(h) > 0.f)) acc[8 * k + 2 * j] = 0.f;
                if (!(__high2float(h) > 0.f)) acc[8 * k + 2 * j + 1] = 0.f;
            }
        }
    }
    uint4 *sw = reinterpret_cast<uint4 *>(stage + warp * 2048);
    const int rx = lane >> 2, kc = lane & 3;  // row phase: pixel in the tile row, 16-byte chunk
    const int own = (lane >> 1) & 3;          // swizzle of this lane's own pixel
    if (a.Y2) {  // the two used channels: 8 B per pixel, a tile row is 64 contiguous bytes
        if (inside) *reinterpret_cast<float2 *>(a.Y2 + (o / C) * 2) = make_float2(acc[0], acc[1]);
        return;
    }
    if (a.Yf) {  // FP32: two halves of 16 channels (64 B per pixel) through the same 2 KB
#pragma unroll
        for (int hf = 0; hf < 2; hf++) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float *q = acc + 16 * hf + 4 * k;
                sw[lane * 4 + (k ^ own)] = make_uint4(__float_as_uint(q[0]), __float_as_uint(q[1]),
                                                      __float_as_uint(q[2]), __float_as_uint(q[3]));
            }
            __syncwarp();
            uint4 v[4];
#pragma unroll
            for (int rr = 0; rr < 4; rr++) {
                const int p = rr * 8 + rx;
                v[rr] = sw[p * 4 + (kc ^ ((p >> 1) & 3))];
            }
            __syncwarp();  // the next half overwrites the slots
#pragma unroll
            for (int rr = 0; rr < 4; rr++) {
                const int ox = x0 + rx, oy = y0 + warp * 4 + rr;
                if (ox < a.W && oy < a.H)
                    *reinterpret_cast<uint4 *>(a.Yf + (((long long)img * a.H + oy) * a.W + ox) * C + 16 * hf +
                                               kc * 4) = v[rr];
            }
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
        sw[lane * 4 + (k ^ own)] = make_uint4(pack2(acc[8 * k], acc[8 * k + 1]), pack2(acc[8 * k + 2], acc[8 * k + 3]),
                                              pack2(acc[8 * k + 4], acc[8 * k + 5]), pack2(acc[8 * k + 6], acc[8 * k + 7]));
    __syncwarp();
    uint4 v[4];  // all four rows read before the first global store
#pragma unroll
    for (int rr = 0; rr < 4; rr++) {
        const int p = rr * 8 + rx;
        v[rr] = sw[p * 4 + (kc ^ ((p >> 1) & 3))];
    }
#pragma unroll
    for (int rr = 0; rr < 4; rr++) {
        const int ox = x0 + rx, oy = y0 + warp * 4 + rr;
        if (ox < a.W && oy < a.H)
            *reinterpret_cast<uint4 *>(a.Ybf + (((long long)img * a.H + oy) * a.W + ox) * C + kc * 8) = v[rr];
    }
}

__global__ void __launch_bounds__(128) conv3x3_fwd_kernel(ConvArgs a, const __grid_constant__ CUtensorMap tmX) {
    extern __shared__ unsigned char sm_raw[];
    unsigned char *sm = smem_align<1024>(sm_raw);
    unsigned char *sW = sm;
    unsigned char *sP0 = sm + kWBytes;  // kFwdBufs patch buffers
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sP0 + kFwdBufs * kPatch);  // [2] MMA done (per TMEM slot)
    uint64_t *full = mbar + 2;                                               // [kFwdBufs] patch loaded
    uint32_t *tslot = reinterpret_cast<uint32_t *>(full + kFwdBufs);
    static_assert((2 + kFwdBufs) * 8 + 4 <= 64, "barriers");
    __shared__ float sBias[32];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const TileGeom G = tile_geom(a.nimg, a.H, a.W);

    // weights -> [tap][quarter][cout] 16-byte rows (K-major B operand)
    for (int c = tid; c < 32 * 36; c += 128) {
        const int n = c / 36, r = c - n * 36;  // r = tap * 4 + quarter
        cp_async16(sW + r * 512 + n * 16, a.Wk + n * KROWS + r * 8, 16);
    }
    cp_async_commit();
    if (tid < 32) sBias[tid] = a.bias ? a.bias[tid] : 0.f;
    if (warp == 0) tmem_alloc(tslot, 64);
    if (tid == 0) {
        for (int k = 0; k < 2 + kFwdBufs; k++) mbar_init(&mbar[k], 1);
        mbar_init_fence();
    }
    cp_async_wait_all();  // the weights
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t id = idesc(128, 32, 0, 0);
    const uint32_t w_u32 = smem_u32(sW);

    // tile t of iteration k -> patch buffer k % kFwdBufs (tid 0)
    auto load = [&](int t, int k) {
        const int img = t / G.per_img, r = t - img * G.per_img;
        const int tyi = r / G.ntx, txi = r - tyi * G.ntx;
        const int b = k % kFwdBufs;
        mbar_expect_tx(&full[b], 4 * kPlaneData);
        issue_patch(&tmX, img, txi * TXP, tyi * TYP, sP0 + b * kPatch, &full[b]);
    };
    int issued = -1, consumed = -1;  // iterations whose load tid 0 issued / waited for
    if (tid == 0 && (int)blockIdx.x < G.total) {
        load(blockIdx.x, 0);
        issued = 0;
    }
    bool failed = false;
    int prev = -1, i = 0;
    for (int t = blockIdx.x;; t += gridDim.x, i++) {
        const bool have = t < G.total;
        // tile i+1 into buffer (i+1) % 3: it held tile i-2, whose MMAs and
        // epilogue finished before the last barrier
        if (have && tid == 0 && t + (int)gridDim.x < G.total) {
            load(t + gridDim.x, i + 1);
            issued = i + 1;
        }
        if (prev >= 0) {  // epilogue of the previous tile overlaps this tile's loads
            const int j = i - 1;
            const bool ok = mbar_wait_first(&mbar[j & 1], (j >> 1) & 1);
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            fence_after();
            // the staging area is the patch buffer of tile j, whose MMAs are done;
            // the next TMA load into it comes after the barrier below (the proxy
            // fence orders these generic accesses before that async write)
            conv_epilogue(a, G, prev, tmem + (uint32_t)((j & 1) * 32), warp, lane, sBias,
                          sP0 + (j % kFwdBufs) * kPatch);
            fence_async_smem();
        }
        if (!have) break;
        fence_before();
        __syncthreads();
        fence_after();
        if (tid == 0 && mbar_wait_first(&full[i % kFwdBufs], (i / kFwdBufs) & 1)) {
            consumed = i;
            const uint32_t p_u32 = smem_u32(sP0 + (i % kFwdBufs) * kPatch);
            const uint32_t d = tmem + (uint32_t)((i & 1) * 32);
#pragma unroll 1
            for (int tap = 0; tap < 9; tap++) {
                const int dy = tap / 3, dx = tap - dy * 3;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const uint64_t da = sdesc(p_u32 + 2 * h * kPlane + (dy * PW + dx) * 16, kPlane, PW * 16);
                    const uint64_t db = sdesc(w_u32 + (tap * 4 + 2 * h) * 512, 512, 128);
                    mma_bf16(d, da, db, id, (tap | h) ? 1u : 0u);
                }
            }
            mma_commit(&mbar[i & 1]);
        }
        prev = t;
    }
    if (failed) {
        if (tid == 0) {
            atomicExch(&g_corr_err, 1);
            // patch loads that may still run: issued but not waited for
            for (int k = consumed + 1; k <= issued; k++) mbar_wait(&full[k % kFwdBufs], (k / kFwdBufs) & 1);
        }
        // the MMAs of the last issued tile may still run
        mbar_wait(&mbar[(i - 1) & 1], ((i - 1) >> 1) & 1);
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) tmem_dealloc(tmem, 64);
}

// Warp-specialised forward convolution (same tiles, operands and epilogue as
// conv3x3_fwd_kernel).  The CTA's tiles are t = blockIdx.x + k * gridDim.x.
//   warp 0 (lane 0): tile k -> patch buffer k % kWsBufs once the MMAs of tile
//     k - kWsBufs have released it (empty barrier), TMA, full barrier;
//   warp 1 (lane 0): waits for the patch and for a free accumulator
//     (tile k - kWsAcc's epilogue has read it), issues the 18 MMAs of tile k
//     into accumulator k % kWsAcc and commits to the patch's empty barrier and
//     the accumulator's full barrier;
//   warps 2-5: wait for the accumulator, read their 32 TMEM lanes (warp w
//     reads lanes 32 (w % 4) ..), release the accumulator, finish the tile.
// No role waits at a CTA barrier inside the loop, so MMAs of tile k run
// while tile k - 1's epilogue stores and tile k + 1..k + 5 load.  Every wait
// is bounded; a role whose wait expires sets the error word and leaves its
// loop, the others' waits then expire in turn, and before TMEM is freed the
// producer waits for its issued-but-unconsumed patch loads and the MMA warp
// for its last MMAs.
__global__ void __launch_bounds__(kWsThreads) conv3x3_fwd_ws_kernel(ConvArgs a, const __grid_constant__ CUtensorMap tmX) {
    extern __shared__ unsigned char sm_raw[];
    unsigned char *sm = smem_align<1024>(sm_raw);
    unsigned char *sW = sm;
    unsigned char *sP0 = sm + kWBytes;                         // kWsBufs patch buffers
    unsigned char *sStage = sP0 + kWsBufs * kPatch;            // 4 x 2 KB epilogue staging
    uint64_t *full = reinterpret_cast<uint64_t *>(sStage + kWsStage);  // [kWsBufs] patch landed
    uint64_t *empty = full + kWsBufs;                                  // [kWsBufs] patch's MMAs done
    uint64_t *accf = empty + kWsBufs;                                  // [kWsAcc] accumulator ready
    uint64_t *acce = accf + kWsAcc;                                    // [kWsAcc] accumulator read
    uint32_t *tslot = reinterpret_cast<uint32_t *>(acce + kWsAcc);
    int *sCount = reinterpret_cast<int *>(tslot + 1);  // [0] loads issued, [1] patches consumed
    __shared__ float sBias[32];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const TileGeom G = tile_geom(a.nimg, a.H, a.W);
    const int ntile = (int)blockIdx.x < G.total ? (G.total - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    for (int c = tid; c < 32 * 36; c += kWsThreads) {
        const int n = c / 36, r = c - n * 36;  // r = tap * 4 + quarter
        cp_async16(sW + r * 512 + n * 16, a.Wk + n * KROWS + r * 8, 16);
    }
    cp_async_commit();
    if (tid < 32) sBias[tid] = a.bias ? a.bias[tid] : 0.f;
    if (warp == 1) tmem_alloc(tslot, 32 * kWsAcc);
    if (tid == 0) {
        for (int k = 0; k < kWsBufs; k++) {
            mbar_init(&full[k], 1);
            mbar_init(&empty[k], 1);
        }
        for (int k = 0; k < kWsAcc; k++) {
            mbar_init(&accf[k], 1);
            mbar_init(&acce[k], 4);  // one arrival per epilogue warp
        }
        sCount[0] = sCount[1] = 0;
        mbar_init_fence();
    }
    cp_async_wait_all();
    fence_async_smem();  // the weights, written by cp.async, are read by the MMAs (async proxy)
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 0) {
        if (lane == 0) {
            int k = 0;
            for (; k < ntile; k++) {
                const int b = k % kWsBufs;
                if (k >= kWsBufs && !mbar_wait_first(&empty[b], ((k / kWsBufs) - 1) & 1)) {
                    atomicExch(&g_corr_err, 1);
                    break;
                }
                const int t = (int)blockIdx.x + k * (int)gridDim.x;
                const int img = t / G.per_img, r = t - img * G.per_img;
                const int tyi = r / G.ntx, txi = r - tyi * G.ntx;
                mbar_expect_tx(&full[b], 4 * kPlaneData);
                issue_patch(&tmX, img, txi * TXP, tyi * TYP, sP0 + b * kPatch, &full[b]);
            }
            sCount[0] = k;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t id = idesc(128, 32, 0, 0);
            const uint32_t w_u32 = smem_u32(sW);
            int k = 0;
            for (; k < ntile; k++) {
                const int b = k % kWsBufs, ac = k % kWsAcc;
                if (!mbar_wait_first(&full[b], (k / kWsBufs) & 1)) {
                    atomicExch(&g_corr_err, 1);
                    break;
                }
                sCount[1] = k + 1;
                if (k >= kWsAcc && !mbar_wait_first(&acce[ac], ((k / kWsAcc) - 1) & 1)) {
                    atomicExch(&g_corr_err, 1);
                    break;
                }
                fence_after();
                const uint32_t p_u32 = smem_u32(sP0 + b * kPatch);
                const uint32_t d = tmem + (uint32_t)(ac * 32);
#pragma unroll 1
                for (int tap = 0; tap < 9; tap++) {
                    const int dy = tap / 3, dx = tap - dy * 3;
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const uint64_t da = sdesc(p_u32 + 2 * h * kPlane + (dy * PW + dx) * 16, kPlane, PW * 16);
                        const uint64_t db = sdesc(w_u32 + (tap * 4 + 2 * h) * 512, 512, 128);
                        mma_bf16(d, da, db, id, (tap | h) ? 1u : 0u);
                    }
                }
                mma_commit(&empty[b]);
                mma_commit(&accf[ac]);
            }
            // the MMAs issued last may still run: they signal the last
            // accumulator's full barrier when done
            if (k > 0) mbar_wait(&accf[(k - 1) % kWsAcc], ((k - 1) / kWsAcc) & 1);
        }
    } else {
        const int q = warp & 3;  // TMEM lane quarter this warp may read
        for (int k = 0; k < ntile; k++) {
            const int ac = k % kWsAcc;
            // every lane waits; the warp leaves together if any lane's wait
            // expired (the TMEM load below is a warp-wide instruction)
            const bool ok = mbar_wait_first(&accf[ac], (k / kWsAcc) & 1);
            if (__any_sync(0xffffffffu, !ok)) {
                if (lane == 0) atomicExch(&g_corr_err, 1);
                break;
            }
            fence_after();
            const int t = (int)blockIdx.x + k * (int)gridDim.x;
            conv_epilogue(a, G, t, tmem + (uint32_t)(ac * 32), q, lane, sBias, sStage, &acce[ac]);
        }
    }
    __syncwarp();
    fence_before();
    __syncthreads();
    if (tid == 0) {  // patch loads issued but never consumed (an expired wait): let them land
        for (int k = sCount[1]; k < sCount[0]; k++) mbar_wait(&full[k % kWsBufs], (k / kWsBufs) & 1);
    }
    __syncthreads();
    fence_after();
    if (warp == 1) tmem_dealloc(tmem, 32 * kWsAcc);
}

// Weight (and bias) gradient partials of this CTA's strip of tiles, written
// to its row of `part` ([gridDim.x][kWgPart]: dW[cout][288], then the 4 warps'
// bias sums [4][32]); wgrad_reduce_kernel adds the rows to dW and db in a
// fixed order, so the gradient does not depend on which CTA finishes first.
constexpr int kWgPart = 32 * KROWS + 4 * 32;
__global__ void __launch_bounds__(128, kWgCtasPerSm)
    conv3x3_wgrad_kernel(const __grid_constant__ CUtensorMap tmXr, const __grid_constant__ CUtensorMap tmZ, int nimg,
                         int H, int W, float *__restrict__ part) {
    extern __shared__ unsigned char sm_raw[];
    unsigned char *sm = smem_align<1024>(sm_raw);  // two stages: patch (12288 B) + dZ planes (4 x 2048 B)
    uint64_t *full = reinterpret_cast<uint64_t *>(sm + 2 * kWgStage);  // [2] stage loaded
    uint64_t *done = full + 2;                                          // [2] MMAs of the stage finished
    uint32_t *tslot = reinterpret_cast<uint32_t *>(full + 4);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const TileGeom G = tile_geom(nimg, H, W);

    if (warp == 0) tmem_alloc(tslot, 128);
    if (tid == 0) {
        for (int k = 0; k < 4; k++) mbar_init(&full[k], 1);
        mbar_init_fence();
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t id = idesc(128, 32, 1, 1);
    const uint32_t sm_u32 = smem_u32(sm);

    // tile t -> stage st: the patch (one 5-D box, zero fill outside the
    // image) and the dZ tile (four channel-quarter boxes)
    auto issue = [&](int t, int st) {
        const int img = t / G.per_img, r = t - img * G.per_img;
        const int tyi = r / G.ntx, txi = r - tyi * G.ntx;
        const int x0 = txi * TXP, y0 = tyi * TYP;
        unsigned char *stg = sm + st * kWgStage;
        mbar_expect_tx(&full[st], kWgPatch + 4 * kZPlane);
        tma_load_5d(stg, &tmXr, 0, x0 - 1, 0, y0 - 1, img, &full[st]);
#pragma unroll
        for (int q = 0; q < 4; q++) tma_load_4d(stg + kWgPatchBuf + q * kZPlane, &tmZ, 8 * q, x0, y0, img, &full[st]);
    };
    // for the error path (tid 0): the last iteration whose load was issued, the
    // last whose load was waited for, and the last whose MMAs were committed
    int last_load = -1, consumed = -1, last_mma = -1;
    if (tid == 0 && (int)blockIdx.x < G.total) {
        issue(blockIdx.x, 0);
        last_load = 0;
    }
    float dbp[8];  // bias gradient partials: cout q * 8 + 2 * (lane & 3) + {0, 1}
#pragma unroll
    for (int k = 0; k < 8; k++) dbp[k] = 0.f;

    bool failed = false;
    int i = 0;
    for (int t = blockIdx.x; t < G.total; t += gridDim.x, i++) {
        const int b = i & 1;
        // first the next tile into the other stage, once the MMAs of the tile
        // it held have finished (its bias reads ended at the last barrier),
        // so that two loads are in flight while this tile waits for its data
        bool ok = true;
        const int tn = t + gridDim.x;
        if (tid == 0 && tn < G.total) {
            if (i >= 1) ok = mbar_wait_first(&done[b ^ 1], ((i - 1) >> 1) & 1);
            if (ok) {
                issue(tn, b ^ 1);
                last_load = i + 1;
            }
        }
        const bool loaded = mbar_wait_first(&full[b], (i >> 1) & 1);
        if (__syncthreads_or(!loaded || !ok)) {
            failed = true;
            break;
        }
        consumed = i;
        if (tid == 0) {
            // D[dy * 32 + cin (+ 32 ignored rows)][cout] for each dx: A = the
            // shifted patch (M groups (dy, quarter) 160 B apart, K groups =
            // tile rows 640 B apart), B = dZ (N groups = quarters, K groups =
            // tile rows 128 B apart); 16 pixels (two tile rows) per MMA
            const uint32_t pb = sm_u32 + b * kWgStage, zb = pb + kWgPatchBuf;
#pragma unroll 1
            for (int s = 0; s < 8; s++) {
                const uint64_t dz = sdesc(zb + s * 256, 128, kZPlane);
#pragma unroll
                for (int dx = 0; dx < 3; dx++) {
                    const uint64_t da = sdesc(pb + s * 2 * kRowQ + dx * 16, kRowQ, PW * 16);
                    mma_bf16(tmem + (uint32_t)(dx * 32), da, dz, id, (i > 0 || s > 0) ? 1u : 0u);
                }
            }
            mma_commit(&done[b]);
            last_mma = i;
        }
        // bias gradient from the dZ tile: per instruction a warp reads 32
        // consecutive words (8 pixels x 16 B), no bank conflicts
        const unsigned char *zt = sm + b * kWgStage + kWgPatchBuf;
#pragma unroll
        for (int q = 0; q < 4; q++) {
#pragma unroll
            for (int pb8 = 0; pb8 < 4; pb8++) {
                const int px = warp * 32 + pb8 * 8 + (lane >> 2);
                const __nv_bfloat162 v =
                    *reinterpret_cast<const __nv_bfloat162 *>(zt + q * kZPlane + px * 16 + (lane & 3) * 4);
                dbp[2 * q] += __low2float(v);
                dbp[2 * q + 1] += __high2float(v);
            }
        }
        fence_async_smem();  // this stage's generic reads before a later TMA write into it
        __syncthreads();
    }
    const int n = i;  // iterations entered (the last may have failed)
    float *prow = part + (size_t)blockIdx.x * kWgPart;
    if (failed || n == 0)  // no partials from this CTA
        for (int k = tid; k < kWgPart; k += 128) prow[k] = 0.f;
    if (failed) {
        if (tid == 0) {
            atomicExch(&g_corr_err, 1);
            // whatever may still run: the last load and the last MMAs
            // loads issued but not waited for (up to two: this tile's and the next)
            for (int k = consumed + 1; k <= last_load; k++) mbar_wait(&full[k & 1], (k >> 1) & 1);
            // the last commit covers every earlier MMA of this thread
            if (last_mma >= 0) mbar_wait(&done[last_mma & 1], (last_mma >> 1) & 1);
        }
    } else if (n > 0) {
        const int L = n - 1;
        const bool ok = mbar_wait_first(&done[L & 1], (L >> 1) & 1);
        if (__syncthreads_or(!ok)) {
            for (int k = tid; k < kWgPart; k += 128) prow[k] = 0.f;
            if (tid == 0) {
                atomicExch(&g_corr_err, 1);
                mbar_wait(&done[L & 1], (L >> 1) & 1);  // the MMAs before TMEM is freed
            }
        } else {
            fence_after();
            if (warp < 3) {  // rows 0..95: dy = warp, cin = lane; rows 96..127 are ignored
#pragma unroll 1
                for (int dx = 0; dx < 3; dx++) {
                    float v[32];
                    tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(dx * 32), v);
                    const int m = (warp * 3 + dx) * 32 + lane;  // tap * 32 + cin
#pragma unroll
                    for (int c = 0; c < 32; c++) prow[c * KROWS + m] = v[c];
                }
            }
#pragma unroll
            for (int k = 0; k < 8; k++) {
                float v = dbp[k];
                v += __shfl_xor_sync(0xffffffffu, v, 4);
                v += __shfl_xor_sync(0xffffffffu, v, 8);
                v += __shfl_xor_sync(0xffffffffu, v, 16);
                dbp[k] = v;
            }
            if (lane < 4) {
                float *pb = prow + 32 * KROWS + warp * 32;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    pb[q * 8 + 2 * lane] = dbp[2 * q];
                    pb[q * 8 + 2 * lane + 1] = dbp[2 * q + 1];
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) tmem_dealloc(tmem, 128);
}

// ---------------------------------------------------------------- training
// Feature scales (metres per unit)
constexpr float kSh = 2.0f;    // maximum depth
constexpr float kSb = 0.05f;   // bed change
constexpr float kSH = 50.0f;   // bathymetry
constexpr float kSdH = 2.0f;   // sub-grid bathymetry detail

// bilinear sample of a coarse [hc][wc] plane at fine cell (x, y), factor f,
// cell-centred, clamped at the edges
__device__ __forceinline__ float up_bilinear(const float *__restrict__ p, int hc, int wc, int f, int x, int y) {
    const float cx = (x + 0.5f) / f - 0.5f, cy = (y + 0.5f) / f - 0.5f;
    const float fx = fminf(fmaxf(cx, 0.f), (float)(wc - 1)), fy = fminf(fmaxf(cy, 0.f), (float)(hc - 1));
    const int x0 = min((int)fx, wc - 1), y0 = min((int)fy, hc - 1);
    const int x1 = min(x0 + 1, wc - 1), y1 = min(y0 + 1, hc - 1);
    const float ax = fx - x0, ay = fy - y0;
    const float a = p[y0 * wc + x0], b = p[y0 * wc + x1], c = p[y1 * wc + x0], d = p[y1 * wc + x1];
    return (1.f - ay) * ((1.f - ax) * a + ax * b) + ay * ((1.f - ax) * c + ax * d);
}

// The network runs on a canvas padded by kPad pixels on each side: a
// padded pixel holds the features of the nearest fine cell (edge
// replication), so that no fine cell is within the 6-layer network's
// receptive radius (6 pixels) of the convolutions' zero padding, which would
// otherwise read as dry, flat land at the image border.  Targets and the
// loss cover the fine cells only.
constexpr int kPad = 8;

struct Canvas {
    int H, W, Hp, Wp;  // fine image, padded canvas
};
__host__ __device__ inline Canvas canvas(int H, int W) { return Canvas{H, W, H + 2 * kPad, W + 2 * kPad}; }
// padded pixel (xp, yp) -> its fine cell (x, y); true if it is that cell
__device__ __forceinline__ bool unpad(const Canvas &cv, int xp, int yp, int &x, int &y) {
    x = min(max(xp - kPad, 0), cv.W - 1);
    y = min(max(yp - kPad, 0), cv.H - 1);
    return x == xp - kPad && y == yp - kPad;
}

// Builds the 32-channel BF16 input of sample idx[b] on the padded canvas
// and, when targets are requested, the normalised residual targets
// T[b][pp][2] (0 outside the fine image); base[b][pp][2] = the interpolated
// coarse maps.
//   coarse: [nsamples][3][hc*wc] = maximum depth, bed change, bathymetry H
//   fineT:  [nsamples][2][H*W]   = maximum depth, bed change (or null)
__global__ void features_kernel(const int *__restrict__ idx, int nb, const float *__restrict__ coarse,
                                const float *__restrict__ fineT, const float *__restrict__ Hf, Canvas cv, int hc,
                                int wc, int f, bf16 *__restrict__ X0, float *__restrict__ T, float *__restrict__ base) {
    const long long npix = (long long)cv.H * cv.W, nppx = (long long)cv.Hp * cv.Wp;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < nb * nppx;
         g += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(g / nppx);
        const long long pp = g - (long long)b * nppx;
        const int yp = (int)(pp / cv.Wp), xp = (int)(pp - (long long)yp * cv.Wp);
        int x, y;
        const bool inside = unpad(cv, xp, yp, x, y);
        const long long p = (long long)y * cv.W + x;
        const int s = idx[b];
        const float *cs = coarse + (long long)s * 3 * hc * wc;
        const float hm = up_bilinear(cs, hc, wc, f, x, y);
        const float dbv = up_bilinear(cs + hc * wc, hc, wc, f, x, y);
        const float Hc = up_bilinear(cs + 2 * hc * wc, hc, wc, f, x, y);
        const float Hfine = Hf[p];
        const int xi = min(x / f, wc - 1), yi = min(y / f, hc - 1);  // coarse cell containing the fine cell
        const float wet = cs[yi * wc + xi] > 0.f ? 1.f : 0.f;
        // channel 5 is 1 everywhere (a bias input); 6 and 7 locate the cell
        // (the source enters through the west boundary)
        const float v[8] = {hm / kSh, dbv / kSb, Hfine / kSH, (Hfine - Hc) / kSdH, wet, 1.f,
                            (float)x / (float)max(cv.W - 1, 1), (float)y / (float)max(cv.H - 1, 1)};
        uint4 *d = reinterpret_cast<uint4 *>(X0 + g * C);
        d[0] = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
        d[1] = d[2] = d[3] = make_uint4(0, 0, 0, 0);
        if (base) {
            base[g * 2] = hm;
            base[g * 2 + 1] = dbv;
        }
        if (T && fineT) {
            const float *ft = fineT + (long long)s * 2 * npix;
            T[g * 2] = inside ? (ft[p] - hm) / kSh : 0.f;
            T[g * 2 + 1] = inside ? (ft[npix + p] - dbv) / kSb : 0.f;
        }
    }
}

// Mean-square loss over the 2 output channels of the fine cells, each
// cell's maximum-depth term weighted by 1 + wbig * T^2 (T: the normalised
// residual target), so that the few large residuals at run-up fronts weigh
// more than their share of cells; dY = d(loss)/d(output) in BF16 (channels
// 2..31 and the padding zero); loss sum accumulated in FP64.
__global__ void loss_kernel(const float *__restrict__ Y, const float *__restrict__ T, int nb, Canvas cv, float wbig,
                            bf16 *__restrict__ dY, double *__restrict__ loss) {
    __shared__ double sred[32];
    const long long nppx = (long long)cv.Hp * cv.Wp;
    const float scale = 1.f / (float)((long long)nb * cv.H * cv.W);  // d/dy of sum(w d^2) / (2 cells)
    double acc = 0.0;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < nb * nppx;
         g += (long long)gridDim.x * blockDim.x) {
        const long long pp = g % nppx;
        const int yp = (int)(pp / cv.Wp), xp = (int)(pp - (long long)yp * cv.Wp);
        int x, y;
        float d0 = 0.f, d1 = 0.f, w0 = 0.f;
        if (unpad(cv, xp, yp, x, y)) {
            const float t0 = T[g * 2];
            w0 = 1.f + wbig * t0 * t0;
            d0 = Y[g * 2] - t0;
            d1 = Y[g * 2 + 1] - T[g * 2 + 1];
            acc += (double)w0 * d0 * d0 + (double)d1 * d1;
        }
        uint4 *gp = reinterpret_cast<uint4 *>(dY + g * C);
        gp[0] = make_uint4(pack2(scale * w0 * d0, scale * d1), 0, 0, 0);
        gp[1] = gp[2] = gp[3] = make_uint4(0, 0, 0, 0);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sred[w];
        atomicAdd(loss, s);
    }
}

// Adam on the FP32 master weights and biases of all layers; refreshes the
// BF16 weights and their tap-flipped transpose (the input-gradient weights:
// Wt[cin][8 - tap][cout] = W[cout][tap][cin]).
__global__ void adam_kernel(float *__restrict__ Wm, float *__restrict__ mW, float *__restrict__ vW,
                            const float *__restrict__ gW, float *__restrict__ Bm, float *__restrict__ mB,
                            float *__restrict__ vB, const float *__restrict__ gB, int nlayers, float lr, float b1,
                            float b2, float c1, float c2, float eps, bf16 *__restrict__ Wbf, bf16 *__restrict__ Wt) {
    const int nw = nlayers * 32 * KROWS;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nw + nlayers * 32; k += gridDim.x * blockDim.x) {
        if (k < nw) {
            const float g = gW[k];
            const float m = b1 * mW[k] + (1.f - b1) * g, v = b2 * vW[k] + (1.f - b2) * g * g;
            mW[k] = m;
            vW[k] = v;
            const float w = Wm[k] - lr * (m / c1) / (sqrtf(v / c2) + eps);
            Wm[k] = w;
            const int l = k / (32 * KROWS), r = k - l * 32 * KROWS, co = r / KROWS, kk = r - co * KROWS;
            const int tap = kk / 32, ci = kk - tap * 32;
            Wbf[k] = __float2bfloat16_rn(w);
            Wt[l * 32 * KROWS + ci * KROWS + (8 - tap) * 32 + co] = __float2bfloat16_rn(w);
        } else {
            const int j = k - nw;
            const float g = gB[j];
            const float m = b1 * mB[j] + (1.f - b1) * g, v = b2 * vB[j] + (1.f - b2) * g * g;
            mB[j] = m;
            vB[j] = v;
            Bm[j] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
        }
    }
}

// Per-cell envelope of the training targets: E[c][p] = max over the batch
// (and earlier batches) of |T[b][p][c]| over the fine cells p.  Non-negative
// floats order like their bit patterns, so the maximum is an integer
// atomicMax.
__global__ void envelope_kernel(const float *__restrict__ T, int nb, Canvas cv, float *__restrict__ E) {
    const long long npix = (long long)cv.H * cv.W;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < nb * npix;
         g += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(g / npix);
        const long long p = g - (long long)b * npix;
        const int y = (int)(p / cv.W), x = (int)(p - (long long)y * cv.W);
        const long long gp = (long long)b * cv.Hp * cv.Wp + (long long)(y + kPad) * cv.Wp + (x + kPad);
        atomicMax(reinterpret_cast<int *>(E) + p, __float_as_int(fabsf(T[gp * 2])));
        atomicMax(reinterpret_cast<int *>(E) + npix + p, __float_as_int(fabsf(T[gp * 2 + 1])));
    }
}

// Corrected fields of one image's fine cells: base + scale * output channel.
// With an envelope E, each channel's residual is first clamped to
// +-k E[c][p], k times the largest residual the training pairs needed at
// that cell.  A maximum depth is not negative (0 = never wet), so the
// corrected one is clipped at 0 when asked.  out = [4][H*W]: corrected
// maximum depth and bed change, then the interpolated ones.
__global__ void apply_kernel(const float *__restrict__ Y, const float *__restrict__ base, Canvas cv, int clip_depth,
                             const float *__restrict__ E, float k, float *__restrict__ out) {
    const long long npix = (long long)cv.H * cv.W;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix;
         p += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(p / cv.W), x = (int)(p - (long long)y * cv.W);
        const long long gp = (long long)(y + kPad) * cv.Wp + (x + kPad);
        float y0 = Y[gp * 2], y1 = Y[gp * 2 + 1];
        if (E) {
            const float e0 = k * E[p], e1 = k * E[npix + p];
            y0 = fminf(fmaxf(y0, -e0), e0);
            y1 = fminf(fmaxf(y1, -e1), e1);
        }
        const float hb = base[gp * 2], bb = base[gp * 2 + 1];
        const float hc = hb + kSh * y0;
        out[p] = clip_depth ? fmaxf(hc, 0.f) : hc;
        out[npix + p] = bb + kSb * y1;
        out[2 * npix + p] = hb;
        out[3 * npix + p] = bb;
    }
}

// tensor map of an NHWC BF16 32-channel tensor [nimg][H][W][32] with boxes of
// 8 channels x bx x by pixels
cudaError_t make_map(CUtensorMap *m, const void *base, int nimg, int H, int W, int bx, int by) {
    EncodeTiledFn f = tensor_map_encoder();
    if (!f) return cudaErrorNotSupported;
    const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)nimg};
    const cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)C * 2 * W, (cuuint64_t)C * 2 * W * H};
    const cuuint32_t box[4] = {8, (cuuint32_t)bx, (cuuint32_t)by, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    const CUresult r = f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(base), dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t prepare() {
    static bool done = false;
    if (done) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(conv3x3_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(conv3x3_fwd_ws_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kWsSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(conv3x3_wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kWgSmem);
    if (e == cudaSuccess) done = true;
    return e;
}

int num_sms() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 148;
    }
    return n;
}

// The warp-specialised forward kernel is the default (8 x 512^2 images, BF16
// output with ReLU: 405 vs 383 TFLOP/s on one box); TSU_CONV_FWD=plain
// selects conv3x3_fwd_kernel, whose four CTAs per SM each alternate MMAs and
// epilogue.
bool fwd_ws() {
    static const bool ws = [] {
        const char *e = std::getenv("TSU_CONV_FWD");
        return !(e && !std::strcmp(e, "plain"));
    }();
    return ws;
}

cudaError_t conv_launch(const ConvArgs &a, cudaStream_t st) {
    cudaError_t e = prepare();
    if (e != cudaSuccess) return e;
    if (reinterpret_cast<uintptr_t>(a.X) % 16) return cudaErrorInvalidValue;
    CUtensorMap mx;
    e = make_map(&mx, a.X, a.nimg, a.H, a.W, PW, PH);
    if (e != cudaSuccess) return e;
    const TileGeom G = tile_geom(a.nimg, a.H, a.W);
    if (fwd_ws()) {  // persistent CTAs, kWsCtasPerSm per SM
        const int ctas = std::min(G.total, kWsCtasPerSm * num_sms());
        conv3x3_fwd_ws_kernel<<<ctas, kWsThreads, kWsSmem, st>>>(a, mx);
        return cudaGetLastError();
    }
    // persistent CTAs, kFwdCtasPerSm per SM (shared memory and TMEM bound)
    const int ctas = std::min(G.total, kFwdCtasPerSm * num_sms());
    conv3x3_fwd_kernel<<<ctas, 128, kFwdSmem, st>>>(a, mx);
    return cudaGetLastError();
}

// The NHWC tensor viewed as [n][y][channel quarter][x][8 channels] (dims
// innermost first: 8 channels, x at 64 B, quarter at 16 B, y, n): a PW x PH
// box lands in shared memory as [row][quarter][x][8], the weight gradient's
// A operand layout.
cudaError_t make_map_rowq(CUtensorMap *m, const void *base, int nimg, int H, int W) {
    EncodeTiledFn f = tensor_map_encoder();
    if (!f) return cudaErrorNotSupported;
    const cuuint64_t dims[5] = {8, (cuuint64_t)W, 4, (cuuint64_t)H, (cuuint64_t)nimg};
    const cuuint64_t strides[4] = {(cuuint64_t)C * 2, 16, (cuuint64_t)C * 2 * W, (cuuint64_t)C * 2 * W * H};
    const cuuint32_t box[5] = {8, (cuuint32_t)PW, 4, (cuuint32_t)PH, 1};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    const CUresult r = f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void *>(base), dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// dW[k] += sum over CTAs b (in order) of part[b][k]; db[n] += sum over b and
// the 4 warps (in order) of the bias partials
__global__ void wgrad_reduce_kernel(const float *__restrict__ part, int nctas, float *__restrict__ dW,
                                    float *__restrict__ db) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < 32 * KROWS) {
        float acc = 0.f;
        for (int b = 0; b < nctas; b++) acc += part[(size_t)b * kWgPart + k];
        dW[k] += acc;
    } else if (db && k < 32 * KROWS + 32) {
        const int n = k - 32 * KROWS;
        float acc = 0.f;
        for (int b = 0; b < nctas; b++)
            for (int w = 0; w < 4; w++) acc += part[(size_t)b * kWgPart + 32 * KROWS + w * 32 + n];
        db[n] += acc;
    }
}

// CTAs of a weight-gradient launch (4 persistent CTAs per SM: 128 TMEM columns each)
int wgrad_ctas(int nimg, int H, int W) { return std::min(tile_geom(nimg, H, W).total, kWgCtasPerSm * num_sms()); }

// part: wgrad_ctas(...) * kWgPart floats of device scratch, or null (then
// allocated on the stream for this call)
cudaError_t wgrad_launch(const bf16 *X, const bf16 *dZ, int nimg, int H, int W, float *dW, float *db, float *part,
                         cudaStream_t st) {
    cudaError_t e = prepare();
    if (e != cudaSuccess) return e;
    if (reinterpret_cast<uintptr_t>(X) % 16 || reinterpret_cast<uintptr_t>(dZ) % 16) return cudaErrorInvalidValue;
    CUtensorMap mx, mz;
    e = make_map_rowq(&mx, X, nimg, H, W);
    if (e == cudaSuccess) e = make_map(&mz, dZ, nimg, H, W, TXP, TYP);
    if (e != cudaSuccess) return e;
    const int ctas = wgrad_ctas(nimg, H, W);
    float *own = nullptr;
    if (!part) {
        e = cudaMallocAsync((void **)&own, (size_t)ctas * kWgPart * sizeof(float), st);
        if (e != cudaSuccess) return e;
        part = own;
    }
    conv3x3_wgrad_kernel<<<ctas, 128, kWgSmem, st>>>(mx, mz, nimg, H, W, part);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
        wgrad_reduce_kernel<<<(32 * KROWS + 32 + 255) / 256, 256, 0, st>>>(part, ctas, dW, db);
        e = cudaGetLastError();
    }
    if (own) {
        const cudaError_t f = cudaFreeAsync(own, st);
        if (e == cudaSuccess) e = f;
    }
    return e;
}

}  // namespace corr

cudaError_t set_wait_limit_corrector(unsigned long long ns) {
    return cudaMemcpyToSymbol(g_wait_limit_ns, &ns, sizeof(ns));
}

}  // namespace tsu

using namespace tsu::corr;

// ------------------------------------------------------------ the corrector
struct TsuCorrector {
    int device = 0;
    int H = 0, W = 0, f = 1, hc = 0, wc = 0, max_batch = 0;
    Canvas cv{};  // the padded canvas the network runs on
    static constexpr int L = 6;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    // parameters
    float *Wm = nullptr, *mW = nullptr, *vW = nullptr, *gW = nullptr;  // [L][32][288]
    float *Bm = nullptr, *mB = nullptr, *vB = nullptr, *gB = nullptr;  // [L][32]
    bf16 *Wbf = nullptr, *Wt = nullptr;
    long adam_t = 0;
    // activations [max_batch][Hp][Wp][32] on the padded canvas: act[0] = features, act[l] = output of layer l-1
    bf16 *act[L] = {};
    float *Yout = nullptr;  // the last layer's output channels 0 and 1 [max_batch][Hp][Wp][2]
    bf16 *g0 = nullptr, *g1 = nullptr;
    float *T = nullptr, *base = nullptr;  // [max_batch][Hp][Wp][2]
    int *d_idx = nullptr;
    double *d_loss = nullptr;
    // data set
    float *Hf = nullptr;                       // fine bathymetry
    float *coarse = nullptr, *fine = nullptr;  // [n][3][hc*wc], [n][2][H*W]
    int nsamples = 0, cap = 0;
    double last_ms = 0.0;
    long last_convs = 0;
    // options (tsu_corr_set_options)
    float wbig = 0.f;
    int clip_depth = 0;
    float envelope = 0.f;
    // per-pixel envelope of the normalised residual targets of samples
    // [0, env_n) ([2][H*W]); ntrain = the training set of the last tsu_corr_train
    float *E = nullptr;
    int env_n = 0, ntrain = 0;
    float *wg_part = nullptr;  // weight-gradient partials of one layer ([CTAs][kWgPart])
};

namespace {
thread_local char g_corr_msg[256] = "";
#define CCK(call)                                                                                \
    do {                                                                                         \
        cudaError_t _e = (call);                                                                 \
        if (_e != cudaSuccess) {                                                                 \
            snprintf(g_corr_msg, sizeof(g_corr_msg), "%s: %s", #call, cudaGetErrorString(_e));   \
            return _e == cudaErrorMemoryAllocation ? TSU_ERR_GPU_OOM : TSU_ERR_CUDA;             \
        }                                                                                        \
    } while (0)

uint64_t splitmix(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double uniform01(uint64_t &s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

void free_all(TsuCorrector *c) {
    float *fp[] = {c->Wm, c->mW, c->vW, c->gW, c->Bm, c->mB, c->vB, c->gB, c->Yout, c->T, c->base, c->Hf, c->coarse, c->fine,
                   c->E, c->wg_part};
    for (float *p : fp) cudaFree(p);
    cudaFree(c->Wbf);
    cudaFree(c->Wt);
    for (bf16 *p : c->act) cudaFree(p);
    cudaFree(c->g0);
    cudaFree(c->g1);
    cudaFree(c->d_idx);
    cudaFree(c->d_loss);
    if (c->e0) cudaEventDestroy(c->e0);
    if (c->e1) cudaEventDestroy(c->e1);
    if (c->st) cudaStreamDestroy(c->st);
}

int upload_weights(TsuCorrector *c, const float *W, const float *B) {
    const int L = TsuCorrector::L;
    const size_t nw = (size_t)L * 32 * KROWS;
    std::vector<bf16> wb(nw), wt(nw);
    for (int l = 0; l < L; l++)
        for (int co = 0; co < 32; co++)
            for (int kk = 0; kk < KROWS; kk++) {
                const size_t k = ((size_t)l * 32 + co) * KROWS + kk;
                const int tap = kk / 32, ci = kk % 32;
                const bf16 v = __float2bfloat16_rn(W[k]);
                wb[k] = v;
                wt[(size_t)l * 32 * KROWS + ci * KROWS + (8 - tap) * 32 + co] = v;
            }
    CCK(cudaMemcpyAsync(c->Wm, W, nw * sizeof(float), cudaMemcpyHostToDevice, c->st));
    CCK(cudaMemcpyAsync(c->Bm, B, (size_t)L * 32 * sizeof(float), cudaMemcpyHostToDevice, c->st));
    CCK(cudaMemcpyAsync(c->Wbf, wb.data(), nw * sizeof(bf16), cudaMemcpyHostToDevice, c->st));
    CCK(cudaMemcpyAsync(c->Wt, wt.data(), nw * sizeof(bf16), cudaMemcpyHostToDevice, c->st));
    CCK(cudaMemsetAsync(c->mW, 0, nw * sizeof(float), c->st));
    CCK(cudaMemsetAsync(c->vW, 0, nw * sizeof(float), c->st));
    CCK(cudaMemsetAsync(c->mB, 0, (size_t)L * 32 * sizeof(float), c->st));
    CCK(cudaMemsetAsync(c->vB, 0, (size_t)L * 32 * sizeof(float), c->st));
    CCK(cudaStreamSynchronize(c->st));
    c->adam_t = 0;
    return TSU_OK;
}

int check_kernel_flag() {
    int flag = 0;
    CCK(cudaMemcpyFromSymbol(&flag, g_corr_err, sizeof(int)));
    if (flag) {
        snprintf(g_corr_msg, sizeof(g_corr_msg), "corrector: a tensor-core wait expired");
        int z = 0;
        cudaMemcpyToSymbol(g_corr_err, &z, sizeof(int));
        return TSU_ERR_CUDA;
    }
    return TSU_OK;
}

// forward pass of `nb` images already in act[0]; the last layer's two used
// output channels in Yout ([pixel][2], FP32)
int forward(TsuCorrector *c, int nb) {
    const int L = TsuCorrector::L;
    for (int l = 0; l < L; l++) {
        ConvArgs a;
        a.X = c->act[l];
        a.nimg = nb;
        a.H = c->cv.Hp;
        a.W = c->cv.Wp;
        a.Wk = c->Wbf + (size_t)l * 32 * KROWS;
        a.bias = c->Bm + l * 32;
        a.relu = (l < L - 1);
        a.gate = nullptr;
        a.Ybf = (l < L - 1) ? c->act[l + 1] : nullptr;
        a.Yf = nullptr;
        a.Y2 = (l < L - 1) ? nullptr : c->Yout;
        CCK(conv_launch(a, c->st));
    }
    return TSU_OK;
}

int load_batch(TsuCorrector *c, const int *idx, int nb, bool targets) {
    CCK(cudaMemcpyAsync(c->d_idx, idx, nb * sizeof(int), cudaMemcpyHostToDevice, c->st));
    features_kernel<<<4 * num_sms(), 256, 0, c->st>>>(c->d_idx, nb, c->coarse, targets ? c->fine : nullptr, c->Hf, c->cv,
                                                      c->hc, c->wc, c->f, c->act[0], targets ? c->T : nullptr,
                                                      c->base);
    CCK(cudaGetLastError());
    return TSU_OK;
}

// the residual envelope of training samples [0, n)
int compute_envelope(TsuCorrector *c, int n) {
    const long long npix = (long long)c->H * c->W;
    CCK(cudaMemsetAsync(c->E, 0, 2 * npix * sizeof(float), c->st));
    std::vector<int> idx(c->max_batch);
    for (int s0 = 0; s0 < n; s0 += c->max_batch) {
        const int nb = std::min(c->max_batch, n - s0);
        for (int b = 0; b < nb; b++) idx[b] = s0 + b;
        const int rc = load_batch(c, idx.data(), nb, true);
        if (rc) return rc;
        envelope_kernel<<<4 * num_sms(), 256, 0, c->st>>>(c->T, nb, c->cv, c->E);
        CCK(cudaGetLastError());
    }
    c->env_n = n;
    return TSU_OK;
}
}  // namespace

extern "C" int tsu_corr_create(TsuCorrector **out, int ny, int nx, int factor, int max_batch, unsigned long long seed,
                               int device) {
    if (!out || ny < 1 || nx < 1 || factor < 1 || ny % factor || nx % factor || max_batch < 1) return TSU_ERR_INVALID;
    *out = nullptr;
    TsuCorrector *c = new (std::nothrow) TsuCorrector();
    if (!c) return TSU_ERR_HOST_OOM;
    c->device = device;
    c->H = ny;
    c->W = nx;
    c->cv = canvas(ny, nx);
    c->f = factor;
    c->hc = ny / factor;
    c->wc = nx / factor;
    c->max_batch = max_batch;
    const int L = TsuCorrector::L;
    const size_t nw = (size_t)L * 32 * KROWS, nbias = (size_t)L * 32;
    const size_t npix = (size_t)max_batch * c->cv.Hp * c->cv.Wp;  // padded canvas
    cudaError_t e = cudaSetDevice(device);
#define CAL(p, bytes) \
    if (e == cudaSuccess) e = cudaMalloc((void **)&(p), (bytes))
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&c->e0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->e1);
    CAL(c->Wm, nw * 4);
    CAL(c->mW, nw * 4);
    CAL(c->vW, nw * 4);
    CAL(c->gW, nw * 4);
    CAL(c->Bm, nbias * 4);
    CAL(c->mB, nbias * 4);
    CAL(c->vB, nbias * 4);
    CAL(c->gB, nbias * 4);
    CAL(c->Wbf, nw * 2);
    CAL(c->Wt, nw * 2);
    for (int l = 0; l < L; l++) CAL(c->act[l], npix * C * 2);
    CAL(c->Yout, npix * 2 * 4);
    CAL(c->g0, npix * C * 2);
    CAL(c->g1, npix * C * 2);
    CAL(c->T, npix * 2 * 4);
    CAL(c->base, npix * 2 * 4);
    CAL(c->d_idx, (size_t)max_batch * 4);
    CAL(c->d_loss, 8);
    CAL(c->Hf, (size_t)ny * nx * 4);
    CAL(c->E, (size_t)2 * ny * nx * 4);
    CAL(c->wg_part, (size_t)wgrad_ctas(max_batch, c->cv.Hp, c->cv.Wp) * kWgPart * 4);
#undef CAL
    if (e == cudaSuccess) e = prepare();
    if (e != cudaSuccess) {
        snprintf(g_corr_msg, sizeof(g_corr_msg), "tsu_corr_create: %s", cudaGetErrorString(e));
        free_all(c);
        delete c;
        return e == cudaErrorMemoryAllocation ? TSU_ERR_GPU_OOM : TSU_ERR_CUDA;
    }
    // He-normal initialisation (SplitMix64 + Box-Muller); the last layer is
    // zero, so the untrained corrector returns the interpolated coarse fields
    std::vector<float> W(nw, 0.f), B(nbias, 0.f);
    uint64_t s = seed;
    const double sd = std::sqrt(2.0 / (9.0 * 32.0));
    for (int l = 0; l < L - 1; l++)
        for (size_t k = 0; k < (size_t)32 * KROWS; k++) {
            const double u1 = uniform01(s), u2 = uniform01(s);
            W[(size_t)l * 32 * KROWS + k] = (float)(sd * std::sqrt(-2.0 * std::log1p(-u1)) * std::cos(2.0 * M_PI * u2));
        }
    int rc = upload_weights(c, W.data(), B.data());
    if (rc) {
        free_all(c);
        delete c;
        return rc;
    }
    *out = c;
    return TSU_OK;
}

extern "C" int tsu_corr_destroy(TsuCorrector *c) {
    if (!c) return TSU_OK;
    cudaSetDevice(c->device);
    if (c->st) cudaStreamSynchronize(c->st);
    free_all(c);
    delete c;
    return TSU_OK;
}

extern "C" int tsu_corr_set_site(TsuCorrector *c, const float *fine_H) {
    if (!c || !fine_H) return TSU_ERR_INVALID;
    CCK(cudaSetDevice(c->device));
    CCK(cudaMemcpyAsync(c->Hf, fine_H, (size_t)c->H * c->W * 4, cudaMemcpyHostToDevice, c->st));
    CCK(cudaStreamSynchronize(c->st));
    return TSU_OK;
}

extern "C" int tsu_corr_add_samples(TsuCorrector *c, int n, const float *coarse, const float *fine) {
    if (!c || n < 1 || !coarse) return TSU_ERR_INVALID;
    CCK(cudaSetDevice(c->device));
    const size_t cs = (size_t)3 * c->hc * c->wc, fs = (size_t)2 * c->H * c->W;
    if (c->nsamples + n > c->cap) {
        const int ncap = std::max(c->nsamples + n, 2 * c->cap);
        float *nc = nullptr, *nf = nullptr;
        CCK(cudaMalloc((void **)&nc, ncap * cs * 4));
        if (cudaMalloc((void **)&nf, ncap * fs * 4) != cudaSuccess) {
            cudaFree(nc);
            snprintf(g_corr_msg, sizeof(g_corr_msg), "tsu_corr_add_samples: out of device memory");
            return TSU_ERR_GPU_OOM;
        }
        if (c->nsamples) {
            CCK(cudaMemcpyAsync(nc, c->coarse, c->nsamples * cs * 4, cudaMemcpyDeviceToDevice, c->st));
            CCK(cudaMemcpyAsync(nf, c->fine, c->nsamples * fs * 4, cudaMemcpyDeviceToDevice, c->st));
        }
        CCK(cudaStreamSynchronize(c->st));
        cudaFree(c->coarse);
        cudaFree(c->fine);
        c->coarse = nc;
        c->fine = nf;
        c->cap = ncap;
    }
    CCK(tsu::bytes_h2d(c->coarse + c->nsamples * cs, coarse, n * cs * 4, c->st));
    if (fine)
        CCK(tsu::bytes_h2d(c->fine + c->nsamples * fs, fine, n * fs * 4, c->st));
    else
        CCK(cudaMemsetAsync(c->fine + c->nsamples * fs, 0, n * fs * 4, c->st));
    CCK(cudaStreamSynchronize(c->st));
    c->nsamples += n;
    return TSU_OK;
}

extern "C" int tsu_corr_num_samples(TsuCorrector *c, int *n) {
    if (!c || !n) return TSU_ERR_INVALID;
    *n = c->nsamples;
    return TSU_OK;
}

extern "C" int tsu_corr_set_options(TsuCorrector *c, float large_residual_weight, int clip_depth, float envelope) {
    if (!c || !(large_residual_weight >= 0.f) || (clip_depth != 0 && clip_depth != 1) || !(envelope >= 0.f))
        return TSU_ERR_INVALID;
    c->wbig = large_residual_weight;
    c->clip_depth = clip_depth;
    c->envelope = envelope;
    return TSU_OK;
}

extern "C" int tsu_corr_get_weights(TsuCorrector *c, float *W, float *B) {
    if (!c || !W || !B) return TSU_ERR_INVALID;
    CCK(cudaSetDevice(c->device));
    CCK(cudaMemcpyAsync(W, c->Wm, (size_t)TsuCorrector::L * 32 * KROWS * 4, cudaMemcpyDeviceToHost, c->st));
    CCK(cudaMemcpyAsync(B, c->Bm, (size_t)TsuCorrector::L * 32 * 4, cudaMemcpyDeviceToHost, c->st));
    CCK(cudaStreamSynchronize(c->st));
    return TSU_OK;
}

extern "C" int tsu_corr_set_weights(TsuCorrector *c, const float *W, const float *B) {
    if (!c || !W || !B) return TSU_ERR_INVALID;
    CCK(cudaSetDevice(c->device));
    return upload_weights(c, W, B);
}

// `iters` Adam steps on mini-batches drawn (seeded) from samples [0, ntrain)
extern "C" int tsu_corr_train(TsuCorrector *c, int ntrain, int iters, int batch, float lr, unsigned long long seed,
                              float *loss) {
    if (!c || ntrain < 1 || ntrain > c->nsamples || iters < 0 || batch < 1 || batch > c->max_batch)
        return TSU_ERR_INVALID;
    CCK(cudaSetDevice(c->device));
    c->ntrain = ntrain;
    const int L = TsuCorrector::L;
    const size_t nw = (size_t)L * 32 * KROWS;
    const long long npix = (long long)batch * c->H * c->W;
    uint64_t s = seed;
    std::vector<int> idx(batch);
    double *h_loss = nullptr;
    CCK(cudaMallocHost((void **)&h_loss, sizeof(double) * std::max(iters, 1)));
    int rc = TSU_OK;
    cudaError_t e = cudaEventRecord(c->e0, c->st);
    for (int it = 0; it < iters && !rc && e == cudaSuccess; it++) {
        for (int b = 0; b < batch; b++) idx[b] = (int)(splitmix(s) % (uint64_t)ntrain);
        rc = load_batch(c, idx.data(), batch, true);
        if (!rc) rc = forward(c, batch);
        if (rc) break;
        e = cudaMemsetAsync(c->d_loss, 0, 8, c->st);
        if (e != cudaSuccess) break;
        loss_kernel<<<4 * num_sms(), 256, 0, c->st>>>(c->Yout, c->T, batch, c->cv, c->wbig, c->g0, c->d_loss);
        if ((e = cudaGetLastError()) != cudaSuccess) break;
        if ((e = cudaMemcpyAsync(h_loss + it, c->d_loss, 8, cudaMemcpyDeviceToHost, c->st)) != cudaSuccess) break;
        if ((e = cudaMemsetAsync(c->gW, 0, nw * 4, c->st)) != cudaSuccess) break;
        if ((e = cudaMemsetAsync(c->gB, 0, (size_t)L * 32 * 4, c->st)) != cudaSuccess) break;
        bf16 *dZ = c->g0, *dX = c->g1;
        for (int l = L - 1; l >= 0 && e == cudaSuccess; l--) {
            e = wgrad_launch(c->act[l], dZ, batch, c->cv.Hp, c->cv.Wp, c->gW + (size_t)l * 32 * KROWS, c->gB + l * 32,
                             c->wg_part, c->st);
            if (e == cudaSuccess && l > 0) {  // dZ_{l-1} = conv(dZ_l, flipped W_l), zero where act[l] <= 0
                ConvArgs a;
                a.X = dZ;
                a.nimg = batch;
                a.H = c->cv.Hp;
                a.W = c->cv.Wp;
                a.Wk = c->Wt + (size_t)l * 32 * KROWS;
                a.bias = nullptr;
                a.relu = 0;
                a.gate = c->act[l];
                a.Ybf = dX;
                a.Yf = nullptr;
                a.Y2 = nullptr;
                e = conv_launch(a, c->st);
                std::swap(dZ, dX);
            }
        }
        if (e != cudaSuccess) break;
        c->adam_t++;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - powf(b1, (float)c->adam_t), c2 = 1.f - powf(b2, (float)c->adam_t);
        adam_kernel<<<(int)((nw + 255) / 256), 256, 0, c->st>>>(c->Wm, c->mW, c->vW, c->gW, c->Bm, c->mB, c->vB, c->gB,
                                                              L, lr, b1, b2, c1, c2, 1e-8f, c->Wbf, c->Wt);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && !rc) e = cudaEventRecord(c->e1, c->st);
    if (e == cudaSuccess && !rc) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess && !rc) {
        snprintf(g_corr_msg, sizeof(g_corr_msg), "tsu_corr_train: %s", cudaGetErrorString(e));
        rc = TSU_ERR_CUDA;
    }
    if (!rc) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->e0, c->e1);
        c->last_ms = ms;
        c->last_convs = (long)iters * (3 * L - 1);
        if (loss)
            for (int it = 0; it < iters; it++) loss[it] = (float)(h_loss[it] / (2.0 * (double)npix));
    }
    cudaFreeHost(h_loss);
    if (rc) return rc;
    return check_kernel_flag();
}

// corrected (and interpolated baseline) fine fields of samples
// [first, first + n): out_* are [n][H][W]; base_* may be null
extern "C" int tsu_corr_predict(TsuCorrector *c, int first, int n, float *out_hmax, float *out_db, float *base_hmax,
                                float *base_db) {
    if (!c || first < 0 || n < 1 || first + n > c->nsamples || !out_hmax || !out_db) return TSU_ERR_INVALID;
    CCK(cudaSetDevice(c->device));
    const size_t np = (size_t)c->H * c->W;
    // the envelope clamp needs the training set's targets (none before training)
    const bool clamp = c->envelope > 0.f && c->ntrain > 0;
    if (clamp && c->env_n != c->ntrain) {
        const int r = compute_envelope(c, c->ntrain);
        if (r) return r;
    }
    float *d_out = nullptr;
    CCK(cudaMalloc((void **)&d_out, 4 * np * 4));
    int rc = TSU_OK;
    for (int k = 0; k < n && !rc; k++) {
        const int s = first + k;
        rc = load_batch(c, &s, 1, false);
        if (!rc) rc = forward(c, 1);
        if (rc) break;
        apply_kernel<<<2 * num_sms(), 256, 0, c->st>>>(c->Yout, c->base, c->cv, c->clip_depth, clamp ? c->E : nullptr,
                                                         c->envelope, d_out);
        float *want[4] = {out_hmax, out_db, base_hmax, base_db};
        void *outs[4];
        const void *ins[4];
        int m = 0;
        for (int q = 0; q < 4; q++)
            if (want[q]) {
                outs[m] = want[q] + k * np;
                ins[m++] = d_out + q * np;
            }
        if (cudaGetLastError() != cudaSuccess ||
            tsu::planes_d2h(m, outs, (size_t)c->W * 4, ins, (size_t)c->W * 4, (size_t)c->W * 4, c->H, c->st) != cudaSuccess ||
            cudaStreamSynchronize(c->st) != cudaSuccess) {
            snprintf(g_corr_msg, sizeof(g_corr_msg), "tsu_corr_predict: CUDA error");
            rc = TSU_ERR_CUDA;
            break;
        }
    }
    cudaFree(d_out);
    if (rc) return rc;
    return check_kernel_flag();
}

// times `iters` forward convolutions of one layer over `nimg` images of the
// first sample's features: device ms per convolution and TFLOP/s
// (2 x pixels x 288 x 32 FLOPs per convolution)
extern "C" int tsu_corr_bench_conv(TsuCorrector *c, int nimg, int iters, double *ms_per_conv, double *tflops) {
    if (!c || nimg < 1 || nimg > c->max_batch || iters < 1 || c->nsamples < 1) return TSU_ERR_INVALID;
    CCK(cudaSetDevice(c->device));
    std::vector<int> idx(nimg, 0);
    int rc = load_batch(c, idx.data(), nimg, false);
    if (rc) return rc;
    ConvArgs a;
    a.X = c->act[0];
    a.nimg = nimg;
    a.H = c->cv.Hp;  // the padded canvas the network runs on
    a.W = c->cv.Wp;
    a.Wk = c->Wbf;
    a.bias = c->Bm;
    a.relu = 1;
    a.gate = nullptr;
    a.Ybf = c->act[1];
    a.Yf = nullptr;
    a.Y2 = nullptr;
    for (int k = 0; k < 3; k++) CCK(conv_launch(a, c->st));
    CCK(cudaEventRecord(c->e0, c->st));
    for (int k = 0; k < iters; k++) CCK(conv_launch(a, c->st));
    CCK(cudaEventRecord(c->e1, c->st));
    CCK(cudaEventSynchronize(c->e1));
    float ms = 0.f;
    CCK(cudaEventElapsedTime(&ms, c->e0, c->e1));
    const double per = ms / iters;
    if (ms_per_conv) *ms_per_conv = per;
    if (tflops) *tflops = 2.0 * nimg * (double)c->cv.Hp * c->cv.Wp * KROWS * 32 / (per * 1e-3) / 1e12;
    return check_kernel_flag();
}

extern "C" int tsu_corr_last_train_ms(TsuCorrector *c, double *ms, long *convs) {
    if (!c || !ms) return TSU_ERR_INVALID;
    *ms = c->last_ms;
    if (convs) *convs = c->last_convs;
    return TSU_OK;
}

// ---- raw kernels on caller-owned device buffers (stream: a cudaStream_t or null)
extern "C" int tsu_corr_conv3x3(const void *X, int nimg, int H, int W, const void *Wk, const float *bias, int relu,
                                const void *gate, void *Ybf, float *Yf, void *stream) {
    if (!X || !Wk || nimg < 1 || H < 1 || W < 1 || (!Ybf && !Yf)) return TSU_ERR_INVALID;
    ConvArgs a;
    a.X = static_cast<const bf16 *>(X);
    a.nimg = nimg;
    a.H = H;
    a.W = W;
    a.Wk = static_cast<const bf16 *>(Wk);
    a.bias = bias;
    a.relu = relu;
    a.gate = static_cast<const bf16 *>(gate);
    a.Ybf = static_cast<bf16 *>(Ybf);
    a.Yf = Yf;
    a.Y2 = nullptr;
    CCK(conv_launch(a, static_cast<cudaStream_t>(stream)));
    return TSU_OK;
}

extern "C" int tsu_corr_conv3x3_wgrad(const void *X, const void *dZ, int nimg, int H, int W, float *dW, float *db,
                                      void *stream) {
    if (!X || !dZ || !dW || nimg < 1 || H < 1 || W < 1) return TSU_ERR_INVALID;
    CCK(wgrad_launch(static_cast<const bf16 *>(X), static_cast<const bf16 *>(dZ), nimg, H, W, dW, db, nullptr,
                     static_cast<cudaStream_t>(stream)));
    return TSU_OK;
}

// synchronises the device and reports (and clears) an expired kernel wait
extern "C" int tsu_corr_status(void) {
    CCK(cudaDeviceSynchronize());
    return check_kernel_flag();
}

extern "C" const char *tsu_corr_last_error(void) { return g_corr_msg; }
