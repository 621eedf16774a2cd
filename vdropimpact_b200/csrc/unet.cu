// A small convolutional U-Net that predicts a correction to the multigrid's
// initial guess, with its training on the GPU.
//
// The network sees the residual r = b - A z0 of the time-extrapolated guess z0
// (normalised by its RMS, on a grid coarsened by an integer factor) and
// predicts delta ~ A^-1 r, the error of z0; z0 + delta starts the V-cycles,
// which still iterate to tolerance. Layers (all 3x3, zero padding, NHWC BF16
// activations, FP32 accumulation, ReLU except the last):
//   L1 16->16, L2 16->16 = e1 | pool | L3 16->32, L4 32->32 = e2 | pool |
//   L5 32->64, L6 64->64 = e3 | pool | L7 64->64, L8 64->64 | up |
//   L9 64->64 (+e3), L10 64->32 | up | L11 32->32 (+e2), L12 32->16 | up |
//   L13 16->16 (+e1), L14 16->16 (linear; channel 0 is the output)
// The input has one channel, padded to 16. Skips are added after the
// convolution of the upsampled tensor, before the ReLU.
//
// Convolutions are implicit GEMMs on the tensor cores (mma.sync m16n8k16,
// BF16 operands, FP32 accumulators): M = pixels (a warp owns 16 pixels of one
// image row), N = output channels, K = 9 taps x input channels. The input
// gradient is the same convolution with flipped, transposed weights; the
// weight gradient is a second GEMM (output channels x input channels over
// pixels) accumulated per CTA and added atomically.
#include "vdi_internal.hh"

#include <cuda_bf16.h>
#include <cstdint>
#include <type_traits>

#include <cmath>
#include <cstring>
#include <vector>

namespace vdi {
namespace unet {

typedef __nv_bfloat16 bf16;

// ------------------------------------------------------------ tensor cores
__device__ __forceinline__ void mma_bf16(float* c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
    return uint32_t(__bfloat16_as_ushort(lo)) | (uint32_t(__bfloat16_as_ushort(hi)) << 16);
}

template <typename T>
__device__ __forceinline__ float to_f(T v);
template <>
__device__ __forceinline__ float to_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ float to_f<bf16>(bf16 v) { return __bfloat162float(v); }

template <typename T>
__device__ __forceinline__ T from_f(float v);
template <>
__device__ __forceinline__ float from_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ bf16 from_f<bf16>(float v) { return __float2bfloat16(v); }

enum { SRC_DIRECT = 0, SRC_UP2 = 1, SRC_POOL2 = 2 };

/** Value of the convolution input at (y,x) of the operating grid (H x W):
 * the source read directly, upsampled x2 (nearest) or pooled 2x2 (mean);
 * zero outside. mask (same shape as the source) zeroes entries whose mask is
 * not positive (the ReLU derivative in the backward pass). */
template <typename TIN>
__device__ __forceinline__ float src_at(const TIN* src, const bf16* mask, int mode, int H, int W, int C, int b, int y,
                                        int x, int c) {
    if (y < 0 || y >= H || x < 0 || x >= W) return 0.f;
    if (mode == SRC_DIRECT) {
        size_t k = ((size_t(b) * H + y) * W + x) * C + c;
        float v = to_f(src[k]);
        return (mask && !(to_f(mask[k]) > 0.f)) ? 0.f : v;
    }
    if (mode == SRC_UP2) {
        int Hs = H >> 1, Ws = W >> 1;
        size_t k = ((size_t(b) * Hs + (y >> 1)) * Ws + (x >> 1)) * C + c;
        return to_f(src[k]);
    }
    int Hs = H * 2, Ws = W * 2;
    float s = 0.f;
    for (int dy = 0; dy < 2; dy++)
        for (int dx = 0; dx < 2; dx++) s += to_f(src[((size_t(b) * Hs + 2 * y + dy) * Ws + 2 * x + dx) * C + c]);
    return 0.25f * s;
}

template <typename TIN, typename TOUT>
struct ConvArgs {
    const TIN* src;        // input source (layout depends on mode)
    const bf16* mask;      // optional ReLU mask for the source (same shape)
    int mode;
    const bf16* w;         // [9][COUT][CIN]
    const float* bias;     // optional [COUT]
    const bf16* resid;     // optional [B][H][W][COUT] added before the activation
    int relu;
    TOUT* out;             // [B][H][W][COUT]
    int B, H, W;
};

constexpr int TPX = 16, TPY = 8;   // pixel tile: 8 rows of 16 pixels, one warp per row

/** 3x3 convolution on the tensor cores. */
template <int CIN, int COUT, typename TIN, typename TOUT>
__global__ void __launch_bounds__(256) conv3x3_k(ConvArgs<TIN, TOUT> a) {
    constexpr int CS = CIN + 8;             // padded pixel stride (bf16) of the input patch
    constexpr int WS = CIN + 8;             // padded stride of a weight row
    constexpr int PW = TPX + 2, PH = TPY + 2;
    extern __shared__ __align__(16) unsigned char smem[];
    bf16* patch = reinterpret_cast<bf16*>(smem);              // [PH][PW][CS]
    bf16* wsm = patch + PH * PW * CS;                         // [9][COUT][WS]
    const int tilesx = (a.W + TPX - 1) / TPX;
    const int bx = blockIdx.x % tilesx, by = blockIdx.x / tilesx;
    const int b = blockIdx.y;
    const int x0 = bx * TPX, y0 = by * TPY;
    for (int t = threadIdx.x; t < PH * PW * CIN; t += blockDim.x) {
        int c = t % CIN, p = t / CIN;
        int px = p % PW, py = p / PW;
        float v = src_at(a.src, a.mask, a.mode, a.H, a.W, CIN, b, y0 + py - 1, x0 + px - 1, c);
        patch[(py * PW + px) * CS + c] = __float2bfloat16(v);
    }
    for (int t = threadIdx.x; t < 9 * COUT * CIN; t += blockDim.x) {
        int c = t % CIN, r = t / CIN;
        wsm[r * WS + c] = a.w[t];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, tq = lane & 3;
    float acc[COUT / 8][4];
#pragma unroll
    for (int n = 0; n < COUT / 8; n++) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
#pragma unroll
    for (int tap = 0; tap < 9; tap++) {
        const int ky = tap / 3, kx = tap % 3;
        const bf16* prow = patch + ((warp + ky) * PW + kx) * CS;   // pixel 0 of this warp's row, shifted by the tap
        const bf16* wt = wsm + tap * COUT * WS;
#pragma unroll
        for (int kc = 0; kc < CIN / 16; kc++) {
            const int k0 = kc * 16 + 2 * tq;
            uint32_t a0 = *reinterpret_cast<const uint32_t*>(prow + g * CS + k0);
            uint32_t a1 = *reinterpret_cast<const uint32_t*>(prow + (g + 8) * CS + k0);
            uint32_t a2 = *reinterpret_cast<const uint32_t*>(prow + g * CS + k0 + 8);
            uint32_t a3 = *reinterpret_cast<const uint32_t*>(prow + (g + 8) * CS + k0 + 8);
#pragma unroll
            for (int n = 0; n < COUT / 8; n++) {
                const bf16* wr = wt + (n * 8 + g) * WS + k0;
                uint32_t b0 = *reinterpret_cast<const uint32_t*>(wr);
                uint32_t b1 = *reinterpret_cast<const uint32_t*>(wr + 8);
                mma_bf16(acc[n], a0, a1, a2, a3, b0, b1);
            }
        }
    }
    const int y = y0 + warp;
    if (y >= a.H) return;
#pragma unroll
    for (int n = 0; n < COUT / 8; n++) {
        const int co = n * 8 + 2 * tq;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int x = x0 + g + 8 * h;
            if (x >= a.W) continue;
            size_t k = ((size_t(b) * a.H + y) * a.W + x) * COUT + co;
            float v0 = acc[n][2 * h], v1 = acc[n][2 * h + 1];
            if (a.bias) {
                v0 += a.bias[co];
                v1 += a.bias[co + 1];
            }
            if (a.resid) {
                v0 += __bfloat162float(a.resid[k]);
                v1 += __bfloat162float(a.resid[k + 1]);
            }
            if (a.relu) {
                v0 = fmaxf(v0, 0.f);
                v1 = fmaxf(v1, 0.f);
            }
            a.out[k] = from_f<TOUT>(v0);
            a.out[k + 1] = from_f<TOUT>(v1);
        }
    }
}

// ------------------------------------------- Blackwell tensor-core path
// The same convolution on the fifth-generation tensor cores (the default
// path; VDI_UNET_TC=0 keeps the mma.sync kernel above): tcgen05.mma with
// both operands in shared memory and the FP32 accumulator in tensor memory.
// One CTA of four warps takes a row segment of TC_M = 128 output pixels
// (the MMA's M), so the A operand of tap (dy, dx) is a window of the staged
// input rows shifted by whole pixels: a pixel's 8-channel chunk is one
// 16-byte core-matrix row, 8 consecutive pixels one 8 x 16-byte core
// matrix, and the operand needs no copy per tap. The weights, already stored
// [tap][cout][cin], are K-major B operands. A CTA stages the weights once and
// then walks a contiguous run of segments, consecutive rows of one segment
// where it can, keeping the input rows in a ring of four: a new segment
// stages one row, while the tensor cores work on the previous one. Each
// segment is 9 * CIN/16 MMAs (K = 16 each) into one accumulator, read back
// with tcgen05.ld for the bias, skip-add, ReLU epilogue.
namespace tc {

constexpr int TC_M = 128;            // output pixels per segment (MMA M)
constexpr int TC_PX = TC_M + 2;      // staged pixels per input row (one halo pixel each side)
constexpr int TC_THREADS = 128;
constexpr int TC_RING = 4;           // staged input rows: three in use, the next being loaded

__device__ int g_timeout;            // set when a bounded wait gave up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

/** Shared-memory matrix descriptor of a K-major operand without swizzle:
 * core matrices of 8 rows x 16 bytes, lbo the byte distance between the two
 * core matrices of one K = 16 step, sbo between consecutive 8-row groups. */
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = uint64_t((addr >> 4) & 0x3FFFu);
    d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
    d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
    d |= uint64_t(1) << 46;          // descriptor version of sm_100
    return d;                         // base offset 0, no swizzle
}

/** Instruction descriptor of kind::f16: BF16 A and B, both K-major, FP32 D,
 * M x N. */
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16_ss(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

/** Waits for the mbarrier phase with a time limit (about 0.5 s of SM
 * clock); false if it gave up. */
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > 1000000000LL) return false;
    }
}

/** 16 consecutive FP32 accumulator columns of this thread's TMEM lane. */
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

/** Dynamic shared memory of conv3x3_tc: the weights and the ring of staged
 * input rows, plus TC_PAD bytes that no descriptor is meant to reach. The pad
 * keeps every address an operand could span inside the CTA's own
 * allocation even if the K and M core-matrix strides were interpreted the
 * other way round (the A operand would then reach 15 x 2080 + 128 bytes
 * past its start): a misread operand gives wrong numbers, which the tests
 * catch, rather than an access outside the CTA's shared memory. */
constexpr size_t TC_PAD = 32 * 1024;
template <int CIN, int COUT>
constexpr size_t tc_smem() {
    return size_t(9) * (CIN / 8) * COUT * 16 + size_t(TC_RING) * (CIN / 8) * TC_PX * 16 + TC_PAD;
}

template <int CIN, int COUT, typename TIN, typename TOUT>
__global__ void __launch_bounds__(TC_THREADS) conv3x3_tc(ConvArgs<TIN, TOUT> a) {
    constexpr int KC = CIN / 8;                              // 16-byte channel chunks
    constexpr uint32_t CHUNKB = uint32_t(TC_PX) * 16;        // one chunk of one staged row
    constexpr uint32_t ROWB = uint32_t(KC) * CHUNKB;         // one staged row, all chunks
    constexpr uint32_t WTAPB = uint32_t(KC) * COUT * 16;     // one tap of weights
    constexpr int TCOLS = COUT < 32 ? 32 : COUT;             // TMEM columns (a power of two, >= 32)
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 256, "tcgen05 shape");
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* wsm = smem;                               // [9][KC][COUT][8] bf16
    unsigned char* rows = smem + 9 * WTAPB;                  // ring [TC_RING][KC][TC_PX][8] bf16
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int q = tid; q < 9 * COUT * KC; q += TC_THREADS) {
        const int kc = q % KC, co = (q / KC) % COUT, t = q / (KC * COUT);
        *reinterpret_cast<uint4*>(wsm + (uint32_t(t) * KC + kc) * COUT * 16 + co * 16) =
            *reinterpret_cast<const uint4*>(a.w + (size_t(t) * COUT + co) * CIN + kc * 8);
    }
    const uint32_t bar_a = smem_u32(&bar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;
    constexpr uint32_t IDESC = idesc_bf16(TC_M, COUT);
    const int segs = (a.W + TC_M - 1) / TC_M;
    // tasks in (segment, image, row) order; each CTA takes a contiguous run,
    // so that consecutive tasks are usually consecutive rows of one segment
    const long tasks = long(a.B) * a.H * segs;
    const long t0 = tasks * blockIdx.x / gridDim.x, t1 = tasks * (blockIdx.x + 1) / gridDim.x;
    // input row yy of image b (pixels x0-1 .. x0+TC_M) into ring slot
    // (yy + 1) % TC_RING, as 16-byte channel chunks
    auto stage = [&](int b, int yy, int x0) {
        unsigned char* dst = rows + uint32_t((yy + 1 + TC_RING) % TC_RING) * ROWB;
        for (int q = tid; q < KC * TC_PX; q += TC_THREADS) {
            const int px = q % TC_PX, kc = q / TC_PX;
            const int xx = x0 + px - 1;
            uint4 v;
            const bool in = yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
            const size_t k8 = ((size_t(b) * a.H + yy) * a.W + xx) * CIN + kc * 8;
            if (std::is_same<TIN, bf16>::value && a.mode == SRC_DIRECT && !a.mask) {
                v = in ? *reinterpret_cast<const uint4*>(a.src + k8) : make_uint4(0, 0, 0, 0);
            } else if (std::is_same<TIN, float>::value && a.mode == SRC_DIRECT) {
                // FP32 source (the input gradient's dY), 8 channels in two
                // 16-byte loads, the ReLU mask as one 16-byte load
                __align__(16) bf16 e[8];
                if (in) {
                    const float4 lo = *reinterpret_cast<const float4*>(reinterpret_cast<const float*>(a.src) + k8);
                    const float4 hi = *reinterpret_cast<const float4*>(reinterpret_cast<const float*>(a.src) + k8 + 4);
                    float f[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
                    if (a.mask) {
                        __align__(16) bf16 mk[8];
                        *reinterpret_cast<uint4*>(mk) = *reinterpret_cast<const uint4*>(a.mask + k8);
#pragma unroll
                        for (int c = 0; c < 8; c++)
                            if (!(__bfloat162float(mk[c]) > 0.f)) f[c] = 0.f;
                    }
#pragma unroll
                    for (int c = 0; c < 8; c++) e[c] = __float2bfloat16(f[c]);
                } else {
#pragma unroll
                    for (int c = 0; c < 8; c++) e[c] = __float2bfloat16(0.f);
                }
                v = *reinterpret_cast<const uint4*>(e);
            } else {
                __align__(16) bf16 e[8];
#pragma unroll
                for (int c = 0; c < 8; c++)
                    e[c] = __float2bfloat16(src_at(a.src, a.mask, a.mode, a.H, a.W, CIN, b, yy, xx, kc * 8 + c));
                v = *reinterpret_cast<const uint4*>(e);
            }
            *reinterpret_cast<uint4*>(dst + uint32_t(kc) * CHUNKB + uint32_t(px) * 16) = v;
        }
    };
    uint32_t phase = 0;
    int ok = 1;
    int pseg = -1, pb = -1, py = -2;   // the previous task, whose next row is staged
    for (long task = t0; task < t1 && ok; task++) {
        const int y = int(task % a.H);
        const long r = task / a.H;
        const int b = int(r % a.B), seg = int(r / a.B), x0 = seg * TC_M;
        if (!(seg == pseg && b == pb && y == py + 1)) {
            stage(b, y - 1, x0);
            stage(b, y, x0);
            stage(b, y + 1, x0);
        }
        fence_async_smem();   // the staged rows (and weights) become visible to the tensor cores
        fence_before();
        __syncthreads();
        fence_after();
        if (tid == 0) {
            uint32_t acc = 0;
#pragma unroll 1
            for (int t = 0; t < 9; t++) {
                const int dy = t / 3, dx = t % 3;
                unsigned char* src_row = rows + uint32_t((y + dy + TC_RING) % TC_RING) * ROWB;   // row y-1+dy
#pragma unroll
                for (int kb = 0; kb < CIN / 16; kb++) {
                    const uint32_t aa = smem_u32(src_row + uint32_t(2 * kb) * CHUNKB + dx * 16);
                    const uint32_t ba = smem_u32(wsm + uint32_t(t) * WTAPB + uint32_t(2 * kb) * COUT * 16);
                    mma_bf16_ss(tmem, sdesc(aa, CHUNKB, 128), sdesc(ba, uint32_t(COUT) * 16, 128), IDESC, acc);
                    acc = 1;
                }
            }
            mma_commit(bar_a);
        }
        // while the tensor cores run: the next task's new row, if it continues
        // this segment, into the ring slot these MMAs do not read (row y-2's)
        if (task + 1 < t1 && y + 1 < a.H) stage(b, y + 2, x0);
        pseg = seg;
        pb = b;
        py = y;
        ok = mbar_wait(bar_a, phase) ? 1 : 0;
        phase ^= 1;
        ok = __syncthreads_and(ok);
        fence_after();
        if (ok) {
            const int x = x0 + warp * 32 + lane;
            const uint32_t ta = tmem + (uint32_t(warp * 32) << 16);
#pragma unroll
            for (int c0 = 0; c0 < COUT; c0 += 16) {
                float v[16];
                tmem_ld16(ta + c0, v);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (x < a.W) {
                    const size_t k = ((size_t(b) * a.H + y) * a.W + x) * COUT + c0;
#pragma unroll
                    for (int c = 0; c < 16; c++) {
                        float w = v[c];
                        if (a.bias) w += a.bias[c0 + c];
                        if (a.resid) w += __bfloat162float(a.resid[k + c]);
                        if (a.relu) w = fmaxf(w, 0.f);
                        a.out[k + c] = from_f<TOUT>(w);
                    }
                }
            }
        }
        fence_before();
        __syncthreads();   // accumulator read and staged rows consumed before the next segment
        fence_after();
    }
    if (!ok) {
        // a wait gave up: note it, and give any MMA still in flight a bounded
        // time to finish before the tensor memory is released
        if (tid == 0) {
            atomicExch(&g_timeout, 1);
            (void)mbar_wait(bar_a, phase ^ 1);
        }
        __syncthreads();
    }
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
}

}  // namespace tc

template <int CIN, int COUT>
constexpr size_t conv_smem() {
    return (size_t(TPY + 2) * (TPX + 2) * (CIN + 8) + size_t(9) * COUT * (CIN + 8)) * sizeof(bf16);
}

/** Weight gradient dW[tap][co][ci] += sum_p G[p][co] X_tap[p][ci] and bias
 * gradient, with G = dY masked by the layer's ReLU (mask = layer output) and
 * X the (resampled) layer input. grid.x CTAs stride over pixel tiles,
 * grid.y = 9 taps. Each CTA accumulates in registers and adds once. */
template <int CIN, int COUT>
__global__ void __launch_bounds__(256) conv_wgrad_k(const bf16* src, int mode, const float* dy, const bf16* ymask,
                                                    float* dw, float* db, int B, int H, int W) {
    constexpr int GS = COUT + 8, XS = CIN + 8;
    constexpr int NPX = TPX * TPY;
    __shared__ __align__(16) bf16 gsm[NPX * GS];
    __shared__ __align__(16) bf16 xsm[NPX * XS];
    const int tap = blockIdx.y, ky = tap / 3 - 1, kx = tap % 3 - 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, tq = lane & 3;
    constexpr int MT = COUT / 16, NT = CIN / 8, TILES = MT * NT;
    constexpr int PER = (TILES + 7) / 8;     // (m,n) tiles per warp
    float acc[PER][4];
#pragma unroll
    for (int q = 0; q < PER; q++) acc[q][0] = acc[q][1] = acc[q][2] = acc[q][3] = 0.f;
    float bacc = 0.f;
    const int tilesx = (W + TPX - 1) / TPX, tilesy = (H + TPY - 1) / TPY, ntiles = tilesx * tilesy * B;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int b = tile / (tilesx * tilesy), r = tile % (tilesx * tilesy);
        const int x0 = (r % tilesx) * TPX, y0 = (r / tilesx) * TPY;
        __syncthreads();
        for (int t = threadIdx.x; t < NPX * COUT; t += blockDim.x) {
            int co = t % COUT, p = t / COUT;
            int x = x0 + p % TPX, y = y0 + p / TPX;
            float v = 0.f;
            if (x < W && y < H) {
                size_t k = ((size_t(b) * H + y) * W + x) * COUT + co;
                v = dy[k];
                if (ymask && !(__bfloat162float(ymask[k]) > 0.f)) v = 0.f;
            }
            gsm[p * GS + co] = __float2bfloat16(v);
        }
        for (int t = threadIdx.x; t < NPX * CIN; t += blockDim.x) {
            int ci = t % CIN, p = t / CIN;
            int x = x0 + p % TPX, y = y0 + p / TPX;
            float v = (x < W && y < H) ? src_at<bf16>(src, nullptr, mode, H, W, CIN, b, y + ky, x + kx, ci) : 0.f;
            xsm[p * XS + ci] = __float2bfloat16(v);
        }
        __syncthreads();
        if (tap == 4 && threadIdx.x < COUT) {
            for (int p = 0; p < NPX; p++) bacc += __bfloat162float(gsm[p * GS + threadIdx.x]);
        }
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int tt = warp + 8 * q;
            if (tt >= TILES) break;
            const int mt = tt / NT, nt = tt % NT;
#pragma unroll
            for (int kc = 0; kc < NPX / 16; kc++) {
                // A = G^T: rows co (mt*16 + ...), cols pixels (kc*16 + ...)
                const int p0 = kc * 16 + 2 * tq;
                const int r0 = mt * 16 + g;
                uint32_t a0 = pack2(gsm[p0 * GS + r0], gsm[(p0 + 1) * GS + r0]);
                uint32_t a1 = pack2(gsm[p0 * GS + r0 + 8], gsm[(p0 + 1) * GS + r0 + 8]);
                uint32_t a2 = pack2(gsm[(p0 + 8) * GS + r0], gsm[(p0 + 9) * GS + r0]);
                uint32_t a3 = pack2(gsm[(p0 + 8) * GS + r0 + 8], gsm[(p0 + 9) * GS + r0 + 8]);
                // B = X: rows pixels, cols ci (nt*8 + g)
                const int c0 = nt * 8 + g;
                uint32_t b0 = pack2(xsm[p0 * XS + c0], xsm[(p0 + 1) * XS + c0]);
                uint32_t b1 = pack2(xsm[(p0 + 8) * XS + c0], xsm[(p0 + 9) * XS + c0]);
                mma_bf16(acc[q], a0, a1, a2, a3, b0, b1);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int tt = warp + 8 * q;
        if (tt >= TILES) break;
        const int mt = tt / NT, nt = tt % NT;
        const int co = mt * 16 + g, ci = nt * 8 + 2 * tq;
        float* d = dw + (size_t(tap) * COUT) * CIN;
        atomicAdd(d + co * CIN + ci, acc[q][0]);
        atomicAdd(d + co * CIN + ci + 1, acc[q][1]);
        atomicAdd(d + (co + 8) * CIN + ci, acc[q][2]);
        atomicAdd(d + (co + 8) * CIN + ci + 1, acc[q][3]);
    }
    if (tap == 4 && threadIdx.x < COUT) atomicAdd(db + threadIdx.x, bacc);
}

/** Flipped, transposed weights for the input gradient:
 * wt[8-tap][ci][co] = w[tap][co][ci]. */
__global__ void flip_transpose_k(const bf16* w, bf16* wt, int cin, int cout) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 9 * cin * cout) return;
    int ci = t % cin, r = t / cin, co = r % cout, tap = r / cout;
    wt[(size_t(8 - tap) * cin + ci) * cout + co] = w[t];
}

/** dsrc += adjoint of the source resampling applied to dx (operating grid
 * H x W, C channels). */
__global__ void resample_adjoint_add_k(const float* dx, float* dsrc, int mode, int B, int H, int W, int C) {
    if (mode == SRC_DIRECT) {
        size_t n = size_t(B) * H * W * C;
        for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x)
            dsrc[k] += dx[k];
        return;
    }
    if (mode == SRC_UP2) {
        int Hs = H >> 1, Ws = W >> 1;
        size_t n = size_t(B) * Hs * Ws * C;
        for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
            int c = k % C;
            size_t p = k / C;
            int xs = p % Ws, ys = (p / Ws) % Hs, b = p / (size_t(Ws) * Hs);
            float s = 0.f;
            for (int dy = 0; dy < 2; dy++)
                for (int dxx = 0; dxx < 2; dxx++) s += dx[((size_t(b) * H + 2 * ys + dy) * W + 2 * xs + dxx) * C + c];
            dsrc[k] += s;
        }
        return;
    }
    int Hs = 2 * H, Ws = 2 * W;
    size_t n = size_t(B) * Hs * Ws * C;
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
        int c = k % C;
        size_t p = k / C;
        int xs = p % Ws, ys = (p / Ws) % Hs, b = p / (size_t(Ws) * Hs);
        dsrc[k] += 0.25f * dx[((size_t(b) * H + ys / 2) * W + xs / 2) * C + c];
    }
}

__global__ void add_f32_k(float* a, const float* b, size_t n) {
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x)
        a[k] += b[k];
}

/** Adam step on FP32 master weights, refreshing the BF16 copy. */
__global__ void adam_k(float* w, bf16* wb, float* g, float* m1, float* m2, size_t n, float lr, float b1, float b2,
                       float c1, float c2, float eps) {
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
        float gv = g[k];
        float a = b1 * m1[k] + (1.f - b1) * gv;
        float v = b2 * m2[k] + (1.f - b2) * gv * gv;
        m1[k] = a;
        m2[k] = v;
        float wv = w[k] - lr * (a / c1) / (sqrtf(v / c2) + eps);
        w[k] = wv;
        if (wb) wb[k] = __float2bfloat16(wv);
        g[k] = 0.f;
    }
}

/** Loss and its gradient on output channel 0: L = mean (y0 - t)^2. */
__global__ void mse_k(const float* y, const float* t, float* dy, int npx, int C, float* loss) {
    __shared__ float ws[32];
    float s = 0.f;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npx; p += gridDim.x * blockDim.x) {
        float d = y[size_t(p) * C] - t[p];
        s += d * d;
        dy[size_t(p) * C] = 2.f * d / npx;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float q = 0.f;
        for (int w = 0; w < int(blockDim.x >> 5); w++) q += ws[w];
        atomicAdd(loss, q / npx);
    }
}

/** Packs a one-channel FP32 image into the 16-channel BF16 network input. */
__global__ void pack_input_k(const float* x, bf16* in, size_t npx) {
    for (size_t p = blockIdx.x * size_t(blockDim.x) + threadIdx.x; p < npx; p += size_t(gridDim.x) * blockDim.x) {
        in[p * 16] = __float2bfloat16(x[p]);
        for (int c = 1; c < 16; c++) in[p * 16 + c] = __float2bfloat16(0.f);
    }
}

__global__ void unpack_output_k(const float* y, float* out, size_t npx) {
    for (size_t p = blockIdx.x * size_t(blockDim.x) + threadIdx.x; p < npx; p += size_t(gridDim.x) * blockDim.x)
        out[p] = y[p * 16];
}

// ---------------------------------------------------------------- host
struct Layer {
    int cin, cout, mode, relu, skip;   // skip: index of the layer whose output is added, or -1
    int src;                           // index of the layer whose output is the input, -1 = network input
    float *w = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;          // [9][cout][cin]
    float *b = nullptr, *gb = nullptr, *bm1 = nullptr, *bm2 = nullptr;       // [cout]
    bf16* wb = nullptr;
    bf16* wt = nullptr;                // flipped, transposed copy for the input gradient
    int H, W;                          // operating grid
};

static const int NL = 14;

struct Net {
    int H, W, Bmax;                    // input grid and batch capacity
    Layer L[NL];
    std::vector<void*> bufs;
    bf16* in = nullptr;                // [B][H][W][16]
    bf16* act[NL];                     // layer outputs (BF16)
    float* outf = nullptr;             // last layer output (FP32)
    float* gact[NL];                   // gradients of layer outputs
    float* gin = nullptr;              // gradient of the network input (discarded)
    float* tmp = nullptr;              // input-gradient scratch (largest layer input)
    float* loss = nullptr;
    int step = 0;
};

/** Whether the forward and input-gradient convolutions run on tcgen05
 * (default) or on mma.sync (VDI_UNET_TC=0), read once per process. */
static bool use_tc() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("VDI_UNET_TC");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v == 1;
}

template <int CIN, int COUT, typename TIN, typename TOUT>
static cudaError_t conv_launch(cudaStream_t s, const ConvArgs<TIN, TOUT>& a) {
    if (use_tc()) {
        // one wave of resident CTAs: each takes a contiguous run of tasks and
        // stages the next rows while its MMAs run
        static int resident = 0;
        if (!resident) {
            cudaError_t e = cudaFuncSetAttribute(tc::conv3x3_tc<CIN, COUT, TIN, TOUT>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 int(tc::tc_smem<CIN, COUT>()));
            if (e != cudaSuccess) return e;
            int dev = 0, sms = 0, per_sm = 0;
            if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
                (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
                (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tc::conv3x3_tc<CIN, COUT, TIN, TOUT>,
                                                                   tc::TC_THREADS, tc::tc_smem<CIN, COUT>())) !=
                    cudaSuccess)
                return e;
            resident = sms * (per_sm > 0 ? per_sm : 1);
        }
        const long tasks = long(a.B) * a.H * ((a.W + tc::TC_M - 1) / tc::TC_M);
        const int grid = int(tasks < resident ? tasks : resident);
        tc::conv3x3_tc<CIN, COUT, TIN, TOUT><<<grid, tc::TC_THREADS, tc::tc_smem<CIN, COUT>(), s>>>(a);
        return cudaGetLastError();
    }
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(conv3x3_k<CIN, COUT, TIN, TOUT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(conv_smem<CIN, COUT>()));
        if (e != cudaSuccess) return e;
        attr = true;
    }
    int tiles = ((a.W + TPX - 1) / TPX) * ((a.H + TPY - 1) / TPY);
    conv3x3_k<CIN, COUT, TIN, TOUT><<<dim3(tiles, a.B), 256, conv_smem<CIN, COUT>(), s>>>(a);
    return cudaGetLastError();
}

template <typename TIN, typename TOUT>
static cudaError_t conv_dispatch(cudaStream_t s, int cin, int cout, const ConvArgs<TIN, TOUT>& a) {
#define VDI_CONV(CI, CO) \
    if (cin == CI && cout == CO) return conv_launch<CI, CO, TIN, TOUT>(s, a);
    VDI_CONV(16, 16) VDI_CONV(16, 32) VDI_CONV(32, 32) VDI_CONV(32, 64) VDI_CONV(64, 64) VDI_CONV(64, 32)
    VDI_CONV(32, 16)
#undef VDI_CONV
    return cudaErrorInvalidValue;
}

static cudaError_t wgrad_dispatch(cudaStream_t s, const Layer& l, const bf16* src, const float* dy, const bf16* ymask,
                                  int B) {
    dim3 grid(148, 9);
#define VDI_WG(CI, CO)                                                                                     \
    if (l.cin == CI && l.cout == CO) {                                                                     \
        conv_wgrad_k<CI, CO><<<grid, 256, 0, s>>>(src, l.mode, dy, ymask, l.g, l.gb, B, l.H, l.W);        \
        return cudaGetLastError();                                                                         \
    }
    VDI_WG(16, 16) VDI_WG(16, 32) VDI_WG(32, 32) VDI_WG(32, 64) VDI_WG(64, 64) VDI_WG(64, 32) VDI_WG(32, 16)
#undef VDI_WG
    return cudaErrorInvalidValue;
}

static int falloc(Net* n, float** p, size_t count) {
    VDI_CUDA(cudaMalloc(p, count * sizeof(float)));
    VDI_CUDA(cudaMemset(*p, 0, count * sizeof(float)));
    n->bufs.push_back(*p);
    return VDI_OK;
}

static int balloc(Net* n, bf16** p, size_t count) {
    VDI_CUDA(cudaMalloc(p, count * sizeof(bf16)));
    VDI_CUDA(cudaMemset(*p, 0, count * sizeof(bf16)));
    n->bufs.push_back(*p);
    return VDI_OK;
}

/** Deterministic initialisation: He-scaled values from a hash of the index. */
static void init_weights(std::vector<float>& w, int fan_in, unsigned seed) {
    double sc = std::sqrt(2.0 / fan_in);
    for (size_t k = 0; k < w.size(); k++) {
        unsigned h = unsigned(k) * 2654435761u ^ (seed * 0x9E3779B9u);
        h ^= h >> 15; h *= 0x2c1b3c6du; h ^= h >> 12; h *= 0x297a2d39u; h ^= h >> 15;
        double u = (h + 0.5) / 4294967296.0;                     // (0,1)
        w[k] = float(sc * std::sqrt(3.0) * (2 * u - 1));         // uniform with the He variance
    }
}

static void net_free(Net* n) {
    for (auto p : n->bufs) cudaFree(p);
    n->bufs.clear();
}

static int net_create(int H, int W, int Bmax, unsigned seed, Net** out) {
    if (H % 8 || W % 16 || H < 8 || W < 16 || Bmax < 1) {
        set_error("unet: grid %dx%d must be a multiple of 8 rows and 16 columns", H, W);
        return VDI_ERR_INVALID_ARGUMENT;
    }
    Net* n = new Net();
    n->H = H; n->W = W; n->Bmax = Bmax;
    // {cin, cout, mode, relu, skip, src}; grid level from the layer position
    const int spec[NL][6] = {{16, 16, 0, 1, -1, -1}, {16, 16, 0, 1, -1, 0},  {16, 32, 2, 1, -1, 1},
                             {32, 32, 0, 1, -1, 2},  {32, 64, 2, 1, -1, 3},  {64, 64, 0, 1, -1, 4},
                             {64, 64, 2, 1, -1, 5},  {64, 64, 0, 1, -1, 6},  {64, 64, 1, 1, 5, 7},
                             {64, 32, 0, 1, -1, 8},  {32, 32, 1, 1, 3, 9},   {32, 16, 0, 1, -1, 10},
                             {16, 16, 1, 1, 1, 11},  {16, 16, 0, 0, -1, 12}};
    const int level[NL] = {0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0};
    int st;
    auto fail = [&](int s) {
        net_free(n);
        delete n;
        return s;
    };
    for (int k = 0; k < NL; k++) {
        Layer& l = n->L[k];
        l.cin = spec[k][0]; l.cout = spec[k][1]; l.mode = spec[k][2]; l.relu = spec[k][3];
        l.skip = spec[k][4]; l.src = spec[k][5];
        l.H = H >> level[k]; l.W = W >> level[k];
        size_t nw = size_t(9) * l.cin * l.cout;
        if ((st = falloc(n, &l.w, nw)) || (st = falloc(n, &l.g, nw)) || (st = falloc(n, &l.m1, nw)) ||
            (st = falloc(n, &l.m2, nw)) || (st = falloc(n, &l.b, l.cout)) || (st = falloc(n, &l.gb, l.cout)) ||
            (st = falloc(n, &l.bm1, l.cout)) || (st = falloc(n, &l.bm2, l.cout)) || (st = balloc(n, &l.wb, nw)) ||
            (st = balloc(n, &l.wt, nw)))
            return fail(st);
        std::vector<float> w(nw);
        init_weights(w, 9 * l.cin, seed + 7919u * k);
        if (k == NL - 1)
            for (auto& v : w) v *= 0.1f;   // start near a zero correction
        std::vector<bf16> wb(nw);
        for (size_t q = 0; q < nw; q++) wb[q] = __float2bfloat16(w[q]);
        if (cudaMemcpy(l.w, w.data(), nw * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(l.wb, wb.data(), nw * 2, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(VDI_ERR_CUDA);
        size_t na = size_t(Bmax) * l.H * l.W * l.cout;
        if ((st = balloc(n, &n->act[k], na)) || (st = falloc(n, &n->gact[k], na))) return fail(st);
    }
    size_t npx = size_t(Bmax) * H * W;
    if ((st = balloc(n, &n->in, npx * 16)) || (st = falloc(n, &n->outf, npx * 16)) ||
        (st = falloc(n, &n->gin, npx * 16)) || (st = falloc(n, &n->tmp, npx * 64)) || (st = falloc(n, &n->loss, 1)))
        return fail(st);
    *out = n;
    return VDI_OK;
}

static const bf16* layer_input(const Net* n, int k) { return n->L[k].src < 0 ? n->in : n->act[n->L[k].src]; }

static int net_forward(Net* n, cudaStream_t s, int B, bool keep_fp32_out) {
    for (int k = 0; k < NL; k++) {
        const Layer& l = n->L[k];
        if (k == NL - 1) {
            ConvArgs<bf16, float> a{layer_input(n, k), nullptr, l.mode, l.wb, l.b, nullptr, 0, n->outf, B, l.H, l.W};
            VDI_CUDA(conv_dispatch(s, l.cin, l.cout, a));
        } else {
            ConvArgs<bf16, bf16> a{layer_input(n, k), nullptr, l.mode, l.wb, l.b,
                                   l.skip >= 0 ? n->act[l.skip] : nullptr, l.relu, n->act[k], B, l.H, l.W};
            VDI_CUDA(conv_dispatch(s, l.cin, l.cout, a));
        }
    }
    (void)keep_fp32_out;
    return VDI_OK;
}

/** d += g where the ReLU mask (the layer output) is positive. */
__global__ void masked_add_k(float* d, const float* g, const bf16* mk, size_t n) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        if (__bfloat162float(mk[i]) > 0.f) d[i] += g[i];
}

/** Backward pass from the gradient in gact[NL-1]; accumulates weight and
 * bias gradients. */
static int net_backward(Net* n, cudaStream_t s, int B) {
    for (int k = 0; k < NL - 1; k++) {
        const Layer& l = n->L[k];
        VDI_CUDA(cudaMemsetAsync(n->gact[k], 0, sizeof(float) * size_t(B) * l.H * l.W * l.cout, s));
    }
    for (int k = NL - 1; k >= 0; k--) {
        const Layer& l = n->L[k];
        const bf16* ymask = l.relu ? n->act[k] : nullptr;
        const float* dy = n->gact[k];
        // skip connection: its gradient is the output gradient through the ReLU
        if (l.skip >= 0) {
            size_t na = size_t(B) * l.H * l.W * l.cout;
            masked_add_k<<<592, 256, 0, s>>>(n->gact[l.skip], dy, ymask, na);
            VDI_CUDA(cudaGetLastError());
        }
        // weight and bias gradients
        VDI_CUDA(wgrad_dispatch(s, l, layer_input(n, k), dy, ymask, B));
        if (k == 0) continue;   // no gradient needed for the network input
        // input gradient on the operating grid, then the resampling adjoint
        int blocks = (9 * l.cin * l.cout + 255) / 256;
        flip_transpose_k<<<blocks, 256, 0, s>>>(l.wb, l.wt, l.cin, l.cout);
        ConvArgs<float, float> a{dy, ymask, SRC_DIRECT, l.wt, nullptr, nullptr, 0, n->tmp, B, l.H, l.W};
        VDI_CUDA(conv_dispatch(s, l.cout, l.cin, a));
        resample_adjoint_add_k<<<592, 256, 0, s>>>(n->tmp, n->gact[l.src], l.mode, B, l.H, l.W, l.cin);
        VDI_CUDA(cudaGetLastError());
    }
    return VDI_OK;
}

}  // namespace unet
}  // namespace vdi

using namespace vdi;
using namespace vdi::unet;

struct vdi_unet {
    Net* net = nullptr;
    cudaStream_t s = nullptr;
};

extern "C" {

int vdi_unet_create(int H, int W, int batch, unsigned seed, void* stream, vdi_unet** out) {
    if (!out) return VDI_ERR_INVALID_ARGUMENT;
    vdi_unet* u = new vdi_unet();
    u->s = static_cast<cudaStream_t>(stream);
    int st = net_create(H, W, batch, seed, &u->net);
    if (st != VDI_OK) {
        delete u;
        return st;
    }
    *out = u;
    return VDI_OK;
}

int vdi_unet_destroy(vdi_unet* u) {
    if (!u) return VDI_OK;
    if (u->net) {
        net_free(u->net);
        delete u->net;
    }
    delete u;
    return VDI_OK;
}

long vdi_unet_param_count(const vdi_unet* u) {
    if (!u) return 0;
    long c = 0;
    for (int k = 0; k < NL; k++) c += 9L * u->net->L[k].cin * u->net->L[k].cout + u->net->L[k].cout;
    return c;
}

/** Reports a tensor-core wait that gave up (the kernels return without
 * their result rather than wait longer). */
static int tc_status(cudaStream_t s) {
    if (!use_tc()) return VDI_OK;
    int t = 0;
    VDI_CUDA(cudaMemcpyFromSymbolAsync(&t, tc::g_timeout, sizeof(int), 0, cudaMemcpyDeviceToHost, s));
    VDI_CUDA(cudaStreamSynchronize(s));
    if (t) {
        set_error("unet: a tensor-core convolution timed out waiting for its MMAs");
        return VDI_ERR_CUDA;
    }
    return VDI_OK;
}

int vdi_unet_tensor_path(void) { return use_tc() ? 1 : 0; }

int vdi_unet_forward(vdi_unet* u, const float* d_in, float* d_out, int batch) {
    if (!u || !d_in || !d_out || batch < 1 || batch > u->net->Bmax) return VDI_ERR_INVALID_ARGUMENT;
    Net* n = u->net;
    size_t npx = size_t(batch) * n->H * n->W;
    pack_input_k<<<592, 256, 0, u->s>>>(d_in, n->in, npx);
    VDI_TRY(net_forward(n, u->s, batch, true));
    unpack_output_k<<<592, 256, 0, u->s>>>(n->outf, d_out, npx);
    VDI_CUDA(cudaGetLastError());
    return tc_status(u->s);
}

int vdi_unet_train_step(vdi_unet* u, const float* d_in, const float* d_target, int batch, float lr, float* loss) {
    if (!u || !d_in || !d_target || batch < 1 || batch > u->net->Bmax) return VDI_ERR_INVALID_ARGUMENT;
    Net* n = u->net;
    cudaStream_t s = u->s;
    size_t npx = size_t(batch) * n->H * n->W;
    pack_input_k<<<592, 256, 0, s>>>(d_in, n->in, npx);
    VDI_TRY(net_forward(n, s, batch, true));
    VDI_CUDA(cudaMemsetAsync(n->loss, 0, sizeof(float), s));
    VDI_CUDA(cudaMemsetAsync(n->gact[NL - 1], 0, sizeof(float) * npx * 16, s));
    mse_k<<<592, 256, 0, s>>>(n->outf, d_target, n->gact[NL - 1], int(npx), 16, n->loss);
    VDI_CUDA(cudaGetLastError());
    VDI_TRY(net_backward(n, s, batch));
    n->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.f - std::pow(b1, float(n->step)), c2 = 1.f - std::pow(b2, float(n->step));
    for (int k = 0; k < NL; k++) {
        Layer& l = n->L[k];
        size_t nw = size_t(9) * l.cin * l.cout;
        adam_k<<<148, 256, 0, s>>>(l.w, l.wb, l.g, l.m1, l.m2, nw, lr, b1, b2, c1, c2, 1e-8f);
        adam_k<<<1, 64, 0, s>>>(l.b, nullptr, l.gb, l.bm1, l.bm2, size_t(l.cout), lr, b1, b2, c1, c2, 1e-8f);
    }
    VDI_CUDA(cudaGetLastError());
    if (loss) {
        VDI_CUDA(cudaMemcpyAsync(loss, n->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
        VDI_CUDA(cudaStreamSynchronize(s));
    }
    return tc_status(s);
}

/** Gradient check support: forward + loss + backward without an update;
 * copies layer k's weight gradient ([9][cout][cin], FP32) and the loss. */
int vdi_unet_gradients(vdi_unet* u, const float* d_in, const float* d_target, int batch, int layer, float* h_grad,
                       float* h_loss) {
    if (!u || layer < 0 || layer >= NL || batch < 1 || batch > u->net->Bmax) return VDI_ERR_INVALID_ARGUMENT;
    Net* n = u->net;
    cudaStream_t s = u->s;
    size_t npx = size_t(batch) * n->H * n->W;
    for (int k = 0; k < NL; k++) {
        Layer& l = n->L[k];
        VDI_CUDA(cudaMemsetAsync(l.g, 0, sizeof(float) * 9 * l.cin * l.cout, s));
        VDI_CUDA(cudaMemsetAsync(l.gb, 0, sizeof(float) * l.cout, s));
    }
    pack_input_k<<<592, 256, 0, s>>>(d_in, n->in, npx);
    VDI_TRY(net_forward(n, s, batch, true));
    VDI_CUDA(cudaMemsetAsync(n->loss, 0, sizeof(float), s));
    VDI_CUDA(cudaMemsetAsync(n->gact[NL - 1], 0, sizeof(float) * npx * 16, s));
    mse_k<<<592, 256, 0, s>>>(n->outf, d_target, n->gact[NL - 1], int(npx), 16, n->loss);
    VDI_TRY(net_backward(n, s, batch));
    Layer& l = n->L[layer];
    VDI_CUDA(cudaMemcpyAsync(h_grad, l.g, sizeof(float) * 9 * l.cin * l.cout, cudaMemcpyDeviceToHost, s));
    VDI_CUDA(cudaMemcpyAsync(h_loss, n->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    VDI_CUDA(cudaStreamSynchronize(s));
    return VDI_OK;
}

/** Copies all parameters (per layer: weights [9][cout][cin] then bias, FP32)
 * to or from host memory. */
int vdi_unet_params(vdi_unet* u, float* h_buf, long count, int to_device) {
    if (!u || !h_buf || count != vdi_unet_param_count(u)) return VDI_ERR_INVALID_ARGUMENT;
    Net* n = u->net;
    long off = 0;
    for (int k = 0; k < NL; k++) {
        Layer& l = n->L[k];
        size_t nw = size_t(9) * l.cin * l.cout;
        if (to_device) {
            VDI_CUDA(cudaMemcpy(l.w, h_buf + off, nw * 4, cudaMemcpyHostToDevice));
            VDI_CUDA(cudaMemcpy(l.b, h_buf + off + nw, l.cout * 4, cudaMemcpyHostToDevice));
            std::vector<bf16> wb(nw);
            for (size_t q = 0; q < nw; q++) wb[q] = __float2bfloat16(h_buf[off + q]);
            VDI_CUDA(cudaMemcpy(l.wb, wb.data(), nw * 2, cudaMemcpyHostToDevice));
        } else {
            VDI_CUDA(cudaMemcpy(h_buf + off, l.w, nw * 4, cudaMemcpyDeviceToHost));
            VDI_CUDA(cudaMemcpy(h_buf + off + nw, l.b, l.cout * 4, cudaMemcpyDeviceToHost));
        }
        off += nw + l.cout;
    }
    return VDI_OK;
}

}  // extern "C"

namespace vdi {
namespace unet {

/** Network input: the residual averaged over factor x factor blocks, divided
 * by its RMS over the fine grid (norm / sqrt(m n)). */
__global__ void restrict_residual_k(const double* __restrict__ r, const double* rnorm, float* in, int m, int n,
                                    int f) {
    const int W = m / f, H = n / f;
    const double rms = *rnorm / sqrt(double(m) * n);
    const double inv = rms > 0 ? 1.0 / (rms * f * f) : 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < W * H; p += gridDim.x * blockDim.x) {
        const int X = p % W, Y = p / W;
        double s = 0;
        for (int dj = 0; dj < f; dj++)
            for (int di = 0; di < f; di++) s += r[(X * f + di) + size_t(m) * (Y * f + dj)];
        in[p] = float(s * inv);
    }
}

/** z += scale * rms * (bilinear prolongation of the network output). */
__global__ void prolong_correction_k(const float* __restrict__ out, const double* rnorm, double* z, int m, int n,
                                     int f, double scale) {
    const int W = m / f, H = n / f;
    const double a = scale * (*rnorm / sqrt(double(m) * n));
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < long(m) * n; k += long(gridDim.x) * blockDim.x) {
        const int i = int(k % m), j = int(k / m);
        float X = (i + 0.5f) / f - 0.5f, Y = (j + 0.5f) / f - 0.5f;
        int I0 = int(floorf(X)), J0 = int(floorf(Y));
        float wx = X - I0, wy = Y - J0;
        int I1 = I0 + 1, J1 = J0 + 1;
        I0 = I0 < 0 ? 0 : (I0 > W - 1 ? W - 1 : I0);
        I1 = I1 < 0 ? 0 : (I1 > W - 1 ? W - 1 : I1);
        J0 = J0 < 0 ? 0 : (J0 > H - 1 ? H - 1 : J0);
        J1 = J1 < 0 ? 0 : (J1 > H - 1 ? H - 1 : J1);
        float v = (1 - wy) * ((1 - wx) * out[I0 + W * J0] + wx * out[I1 + W * J0]) +
                  wy * ((1 - wx) * out[I0 + W * J1] + wx * out[I1 + W * J1]);
        z[k] += a * double(v);
    }
}

}  // namespace unet

int unet_correct(vdi_unet* u, cudaStream_t s, const double* r, const double* d_rnorm, double* z, int m, int n,
                 int factor, double scale, float* in_buf, float* out_buf) {
    using namespace unet;
    Net* net = u->net;
    if (m / factor != net->W || n / factor != net->H) {
        set_error("unet: grid %dx%d / %d does not match the network's %dx%d", m, n, factor, net->W, net->H);
        return VDI_ERR_INVALID_ARGUMENT;
    }
    restrict_residual_k<<<592, 256, 0, s>>>(r, d_rnorm, in_buf, m, n, factor);
    size_t npx = size_t(net->H) * net->W;
    pack_input_k<<<592, 256, 0, s>>>(in_buf, net->in, npx);
    VDI_TRY(net_forward(net, s, 1, true));
    unpack_output_k<<<592, 256, 0, s>>>(net->outf, out_buf, npx);
    prolong_correction_k<<<1184, 256, 0, s>>>(out_buf, d_rnorm, z, m, n, factor, scale);
    VDI_CUDA(cudaGetLastError());
    return VDI_OK;
}

int unet_kernels_per_correction() {
    return 4 + unet::NL;   // restrict, pack, one per layer, unpack, prolong
}

int unet_dims(const vdi_unet* u, int* H, int* W) {
    *H = u->net->H;
    *W = u->net->W;
    return VDI_OK;
}

}  // namespace vdi
