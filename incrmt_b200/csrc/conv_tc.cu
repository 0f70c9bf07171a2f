// tcgen05 implicit-GEMM convolutions (see conv_tc.cuh).
//
// One CTA of 128 threads computes a 128-pixel x Cout tile of the output:
//  - warp 0, one thread: TMA producer. For every (tap, channel chunk) it
//    loads the tile's input pixels shifted by the tap, [128 pixels][KC
//    channels], from a 4-D tensor map over the NHWC activations (the shift
//    goes into the W and H coordinates; TMA fills pixels outside the image
//    with zeros, which is the convolution's zero padding) and the weights
//    [Cout][KC] of that tap and chunk, into one stage of a ring of shared
//    memory buffers, both with the swizzle that matches KC (32, 64 or 128
//    byte rows).
//  - warp 1, one thread: issues tcgen05.mma (kind::f16, BF16 operands, FP32
//    accumulator in tensor memory, M = 128, N = Cout, K = 16 per
//    instruction) on each stage and releases the stage with tcgen05.commit.
//  - all four warps: epilogue. Each warp reads its 32 tensor-memory lanes
//    (one pixel per thread) with tcgen05.ld, adds the bias, applies the
//    ReLU and stores BF16.
// Every wait on a barrier gives up after one second (%globaltimer), sets
// g_conv_timeout and lets the CTA finish: the producer then waits, again
// bounded, for its loads in flight, the MMA thread still commits so that the
// epilogue only reads after the issued MMAs are done, and tensor memory is
// freed before the CTA exits.
#include <cstdint>
#include <cstring>
#include "common.cuh"
#include "conv_tc.cuh"

namespace incrmt {

__device__ int g_conv_timeout = 0;

namespace {

using bf16 = __nv_bfloat16;

constexpr int kThreads = 128;
constexpr int kTileM = 128;
constexpr int kRowsW = 16, kRowsH = 8;  // the tile of the row-reuse kernel
static_assert(kRowsW * kRowsH == kTileM && kRowsW % 8 == 0, "row-reuse tile: 128 pixels, whole swizzle groups");
constexpr unsigned long long kWaitNs = 1000000000ull;  // one second

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

/** Waits for the phase of parity `parity` of the barrier to complete, at
 * most one second; false (and the timeout flag set) if it did not. */
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_test(bar, parity)) {
        if (global_ns() - t0 > kWaitNs) {
            atomicExch(&g_conv_timeout, 1);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int c0, int c1,
                                            int c2, int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int c0, int c1,
                                            int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

/** Shared-memory matrix descriptor of a K-major operand tile whose rows
 * (one per M or N index) are KC BF16 = 2*KC bytes with the matching swizzle
 * (32, 64 or 128 bytes), eight-row groups 16*KC bytes apart. */
template <int KC>
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    constexpr uint64_t layout = KC == 64 ? 2 : KC == 32 ? 4 : 6;  // SWIZZLE_128B / 64B / 32B
    constexpr uint64_t sbo = (8 * 2 * KC) >> 4;
    return static_cast<uint64_t>((addr >> 4) & 0x3FFF) | (1ull << 16) | (sbo << 32) | (1ull << 46) | (layout << 61);
}

/** Instruction descriptor of kind::f16: BF16 A and B, both K-major, FP32
 * accumulator, M = 128, N = n. */
__host__ __device__ constexpr uint32_t instr_desc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(
            tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

/** Sixteen consecutive 32-bit columns of this thread's tensor-memory lane. */
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

/** The convolution kernel (see the file comment); blockIdx.y selects the
 * output channels n0 = N * blockIdx.y .. n0 + N - 1 of ldy. Dynamic shared
 * memory: 1024 (alignment) + S stage buffers, then 2S + 1 barriers (full[S],
 * empty[S], done) and the tensor-memory address.
 *
 * ROWS (3x3 only, Wt = 16, Ht = 8): a stage holds, for one column offset dx
 * and channel chunk, the (Ht + 2) x Wt input pixels of the tile's rows -1 ..
 * Ht shifted by dx (one TMA load) and the weights of the three taps of that
 * column; the three row offsets dy are the same buffer read Wt, i.e. a whole
 * number of eight-row swizzle groups, further on. Each input pixel then
 * crosses from L2 3 (Ht + 2) / Ht = 3.75 times instead of 9, and each barrier
 * round trip feeds three times the tensor-core work. Otherwise a stage holds
 * one tap: 128 shifted pixels and that tap's weights. */
template <int TAPS, int KC, bool ROWS, int HALVES = 1>
__global__ void __launch_bounds__(kThreads, 1)
    k_conv_tc(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
              const float *__restrict__ bias, bf16 *__restrict__ Y, int H, int W, int N, int ldy, int Wt, int Ht,
              int tiles_x, int tiles_y, int nck, int flip, int relu, int S, uint32_t tmem_cols) {
    static_assert(!ROWS || TAPS == 9, "row reuse is for 3x3 convolutions");
    static_assert(HALVES == 1 || ROWS, "two halves only with row reuse");
    // HALVES = 2 (row reuse): the tile is 16 x 16 pixels, two 128-pixel
    // halves stacked in y, each with its own tensor-memory accumulator of
    // tmem_cols / 2 columns; a stage holds the 16 x 18 input pixels of both
    // (rows -1 .. 16) and the three taps' weights, which both halves use.
    constexpr int kGroup = ROWS ? 3 : 1;                         // taps per stage
    constexpr uint32_t abytes = (ROWS ? HALVES * kTileM + 2 * kRowsW : kTileM) * KC * 2;
    extern __shared__ __align__(1024) unsigned char conv_smem[];
    const uint32_t raw = smem_addr(conv_smem);
    const uint32_t base = (raw + 1023u) & ~1023u;
    const uint32_t tbytes = static_cast<uint32_t>(N) * KC * 2, bbytes = kGroup * tbytes;
    const uint32_t sA = base, sB = base + S * abytes;
    const uint32_t bar0 = sB + S * bbytes;  // full[s] = bar0 + 8s, empty[s] = bar0 + 8(S+s), done = bar0 + 16S
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(conv_smem + (bar0 + 8 * (2 * S + 1) - raw));
    const uint32_t done = bar0 + 16 * S;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int tile = blockIdx.x;
    const int tx = tile % tiles_x;
    tile /= tiles_x;
    const int ty = tile % tiles_y, b = tile / tiles_y;
    const int x0 = tx * Wt, y0 = ty * Ht, n0 = blockIdx.y * N;

    if (threadIdx.x == 0) {
        for (int q = 0; q < 2 * S + 1; q++) mbar_init(bar0 + 8 * q, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapA)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapB)) : "memory");
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int iters = (TAPS / kGroup) * nck;

    if (threadIdx.x == 0) {
        // TMA producer
        int issued = 0;
        for (int it = 0; it < iters; it++) {
            const int s = it % S;
            if (it >= S && !mbar_wait(bar0 + 8 * (S + s), ((it / S) - 1) & 1)) break;
            const int g = it / nck, ck = it - g * nck;
            const uint32_t full = bar0 + 8 * s;
            mbar_arrive_expect_tx(full, abytes + bbytes);
            if constexpr (ROWS) {
                // column offset g - 1; rows -1 .. Ht of the tile
                tma_load_4d(sA + s * abytes, &mapA, full, ck * KC, x0 + g - 1, y0 - 1, b);
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    const int tap = 3 * r + g;
                    tma_load_3d(sB + s * bbytes + r * tbytes, &mapB, full, ck * KC, n0, flip ? 8 - tap : tap);
                }
            } else {
                const int tap = g;
                const int dy = TAPS == 9 ? tap / 3 - 1 : 0, dx = TAPS == 9 ? tap % 3 - 1 : 0;
                tma_load_4d(sA + s * abytes, &mapA, full, ck * KC, x0 + dx, y0 + dy, b);
                tma_load_3d(sB + s * bbytes, &mapB, full, ck * KC, n0, flip ? TAPS - 1 - tap : tap);
            }
            issued = it + 1;
        }
        // No copy may still be in flight when the CTA exits: wait for the last
        // use of every stage (at once when the MMA thread consumed it).
        for (int it = issued > S ? issued - S : 0; it < issued; it++) mbar_wait(bar0 + 8 * (it % S), (it / S) & 1);
    } else if (threadIdx.x == 32) {
        // MMA issuer
        const uint32_t idesc = instr_desc(N);
        for (int it = 0; it < iters; it++) {
            const int s = it % S;
            if (!mbar_wait(bar0 + 8 * s, (it / S) & 1)) break;
            tc_fence_after();
#pragma unroll
            for (int h = 0; h < HALVES; h++)
#pragma unroll
                for (int r = 0; r < kGroup; r++) {
                    // row offset r - 1: the stage's pixels from row h * 8 + r on (ROWS)
                    const uint64_t ad = smem_desc<KC>(sA + s * abytes + (h * kRowsH + r) * kRowsW * KC * 2),
                                   bd = smem_desc<KC>(sB + s * bbytes + r * tbytes);
#pragma unroll
                    for (int k = 0; k < KC / 16; k++)
                        tc_mma(tmem + h * (tmem_cols / HALVES), ad + 2 * k, bd + 2 * k, idesc,
                               (it > 0 || r > 0 || k > 0) ? 1u : 0u);
                }
            tc_commit(bar0 + 8 * (S + s));
        }
        // arrives once every MMA issued above has completed
        tc_commit(done);
    }
    __syncwarp();

    // Epilogue: warp w holds tensor-memory lanes 32w..32w+31, the tile's
    // pixels in row-major order of the Wt x Ht tile.
    bool ok = mbar_wait(done, 0);
    // the tensor-memory loads below are warp-collective: converge, and agree
    // on whether the wait succeeded
    ok = __all_sync(0xffffffffu, ok);
    tc_fence_after();
    for (int h = 0; h < HALVES && ok; h++) {
        const int r = warp * 32 + lane;
        const int py = y0 + h * kRowsH + r / Wt, px = x0 + r % Wt;
        const bool valid = py < H && px < W;
        bf16 *yrow = Y + ((static_cast<long>(b) * H + py) * W + px) * static_cast<long>(ldy) + n0;
        for (int c0 = 0; c0 < N; c0 += 16) {
            uint32_t v[16];
            tc_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + h * (tmem_cols / HALVES) +
                        static_cast<uint32_t>(c0),
                    v);
            if (!valid) continue;
            uint32_t packed[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                float f0 = __uint_as_float(v[2 * j]), f1 = __uint_as_float(v[2 * j + 1]);
                if (bias) {
                    f0 += bias[n0 + c0 + 2 * j];
                    f1 += bias[n0 + c0 + 2 * j + 1];
                }
                if (relu) {
                    f0 = fmaxf(f0, 0.f);
                    f1 = fmaxf(f1, 0.f);
                }
                const __nv_bfloat162 hv = __floats2bfloat162_rn(f0, f1);
                packed[j] = *reinterpret_cast<const uint32_t *>(&hv);
            }
            uint4 *dst = reinterpret_cast<uint4 *>(yrow + c0);
            dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
            dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols) : "memory");
}

constexpr int kPersistThreads = 192;  // producer warp, MMA warp, four epilogue warps

/** Persistent 3x3 convolution with the layer's weights resident in shared
 * memory (row reuse as in k_conv_tc<9, KC, true>). Each CTA loads all 9 x
 * Cin x N weights once, then walks the 16 x 8 pixel tiles blockIdx.x,
 * blockIdx.x + gridDim.x, ...: warp 0 (one thread) streams the tiles' input
 * stages (one column offset and channel chunk each: 16 x 10 pixels x KC)
 * through a ring of S buffers without draining between tiles, warp 1 (one
 * thread) issues the three row offsets' MMAs of each stage against the
 * resident weights into one of two tensor-memory accumulators (tile j uses
 * accumulator j mod 2), and warps 2-5 drain the other accumulator (bias,
 * ReLU, BF16 stores) while the next tile accumulates. Only input pixels cross
 * from L2 per tile. Barriers: full[S], empty[S] (stage ring), wfull
 * (weights), tfull[2] (MMA -> epilogue), tempty[2] (epilogue -> MMA, one
 * arrival per epilogue warp), done (all MMAs complete). Every wait is
 * bounded as in k_conv_tc. Dynamic shared memory: 1024 + W + S * A + 8 *
 * (2S + 6) + 16, W = 9 (Cin / KC) N KC 2 bytes of weights, A = 160 KC 2. */
template <int KC>
__global__ void __launch_bounds__(kPersistThreads, 1)
    k_conv_tc_persist(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                      const float *__restrict__ bias, bf16 *__restrict__ Y, int H, int W, int N, int tiles_x,
                      int tiles_y, int ntiles, int nck, int flip, int relu, int S, uint32_t cols) {
    constexpr uint32_t abytes = (kTileM + 2 * kRowsW) * KC * 2;
    extern __shared__ __align__(1024) unsigned char conv_smem[];
    const uint32_t raw = smem_addr(conv_smem);
    const uint32_t base = (raw + 1023u) & ~1023u;
    const uint32_t tbytes = static_cast<uint32_t>(N) * KC * 2;  // one (tap, chunk) block of weights
    const uint32_t wbytes = 9u * nck * tbytes;
    const uint32_t sW = base, sA = base + wbytes;
    const uint32_t bar0 = sA + S * abytes;
    // full[s] = bar0 + 8s, empty[s] = bar0 + 8(S+s), then wfull, tfull[2], tempty[2], done
    const uint32_t wfull = bar0 + 16 * S, tfull = wfull + 8, tempty = tfull + 16, done = tempty + 16;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(conv_smem + (done + 8 - raw));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int G = gridDim.x;

    if (threadIdx.x == 0) {
        for (int q = 0; q < 2 * S; q++) mbar_init(bar0 + 8 * q, 1);
        mbar_init(wfull, 1);
        mbar_init(tfull, 1);
        mbar_init(tfull + 8, 1);
        mbar_init(tempty, 4);
        mbar_init(tempty + 8, 4);
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapA)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapB)) : "memory");
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(2 * cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (threadIdx.x == 0) {
        // producer: the weights once, then the tiles' input stages
        mbar_arrive_expect_tx(wfull, wbytes);
        for (int tap = 0; tap < 9; tap++)
            for (int ck = 0; ck < nck; ck++)
                tma_load_3d(sW + (tap * nck + ck) * tbytes, &mapB, wfull, ck * KC, 0, flip ? 8 - tap : tap);
        int it = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += G) {
            int t = tile;
            const int tx = t % tiles_x;
            t /= tiles_x;
            const int ty = t % tiles_y, b = t / tiles_y;
            const int x0 = tx * kRowsW, y0 = ty * kRowsH;
            for (int g = 0; g < 3 && ok; g++)
                for (int ck = 0; ck < nck; ck++) {
                    const int s = it % S;
                    if (it >= S && !mbar_wait(bar0 + 8 * (S + s), ((it / S) - 1) & 1)) { ok = false; break; }
                    mbar_arrive_expect_tx(bar0 + 8 * s, abytes);
                    tma_load_4d(sA + s * abytes, &mapA, bar0 + 8 * s, ck * KC, x0 + g - 1, y0 - 1, b);
                    it++;
                }
        }
        // no copy may still be in flight when the CTA exits
        for (int q = it > S ? it - S : 0; q < it; q++) mbar_wait(bar0 + 8 * (q % S), (q / S) & 1);
        mbar_wait(wfull, 0);
    } else if (threadIdx.x == 32) {
        // MMA issuer
        const uint32_t idesc = instr_desc(N);
        bool ok = mbar_wait(wfull, 0);
        int it = 0, j = 0;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += G, j++) {
            const int a = j & 1;
            if (j >= 2 && !mbar_wait(tempty + 8 * a, ((j >> 1) - 1) & 1)) break;
            tc_fence_after();
            const uint32_t acc = tmem + a * cols;
            for (int g = 0; g < 3 && ok; g++)
                for (int ck = 0; ck < nck; ck++) {
                    const int s = it % S;
                    if (!mbar_wait(bar0 + 8 * s, (it / S) & 1)) { ok = false; break; }
                    tc_fence_after();
#pragma unroll
                    for (int r = 0; r < 3; r++) {
                        const uint64_t ad = smem_desc<KC>(sA + s * abytes + r * kRowsW * KC * 2),
                                       bd = smem_desc<KC>(sW + ((3 * r + g) * nck + ck) * tbytes);
#pragma unroll
                        for (int k = 0; k < KC / 16; k++)
                            tc_mma(acc, ad + 2 * k, bd + 2 * k, idesc, (g > 0 || ck > 0 || r > 0 || k > 0) ? 1u : 0u);
                    }
                    tc_commit(bar0 + 8 * (S + s));
                    it++;
                }
            tc_commit(tfull + 8 * a);
        }
        // arrives once every MMA issued above has completed
        tc_commit(done);
    } else if (warp >= 2) {
        // epilogue: warp w reads tensor-memory lanes 32 (w mod 4) .. + 31
        const int q = warp & 3;
        const int r = q * 32 + lane;
        int j = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += G, j++) {
            const int a = j & 1;
            bool ok = mbar_wait(tfull + 8 * a, (j >> 1) & 1);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) break;
            tc_fence_after();
            int t = tile;
            const int tx = t % tiles_x;
            t /= tiles_x;
            const int ty = t % tiles_y, b = t / tiles_y;
            const int py = ty * kRowsH + r / kRowsW, px = tx * kRowsW + r % kRowsW;
            const bool valid = py < H && px < W;
            bf16 *yrow = Y + ((static_cast<long>(b) * H + py) * W + px) * static_cast<long>(N);
            for (int c0 = 0; c0 < N; c0 += 16) {
                uint32_t v[16];
                tc_ld16(tmem + (static_cast<uint32_t>(q * 32) << 16) + a * cols + static_cast<uint32_t>(c0), v);
                if (!valid) continue;
                uint32_t packed[8];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    float f0 = __uint_as_float(v[2 * e]), f1 = __uint_as_float(v[2 * e + 1]);
                    if (bias) {
                        f0 += bias[c0 + 2 * e];
                        f1 += bias[c0 + 2 * e + 1];
                    }
                    if (relu) {
                        f0 = fmaxf(f0, 0.f);
                        f1 = fmaxf(f1, 0.f);
                    }
                    const __nv_bfloat162 h = __floats2bfloat162_rn(f0, f1);
                    packed[e] = *reinterpret_cast<const uint32_t *>(&h);
                }
                uint4 *dst = reinterpret_cast<uint4 *>(yrow + c0);
                dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
                dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty + 8 * a);
        }
    }
    __syncwarp();
    if (warp == 0) {
        // every MMA done before the tensor memory is freed
        mbar_wait(done, 0);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * cols) : "memory");
}

/** Shared-memory descriptor of an MN-major operand: atoms of KA elements
 * along M or N (rows of 2*KA bytes, the matching swizzle) for every pixel,
 * eight pixels per 8*2*KA-byte swizzle group (SBO), atoms `lbo` bytes
 * apart (LBO). */
template <int KA>
__device__ __forceinline__ uint64_t smem_desc_mn(uint32_t addr, uint32_t lbo) {
    constexpr uint64_t layout = KA == 64 ? 2 : KA == 32 ? 4 : 6;
    constexpr uint64_t sbo = (8 * 2 * KA) >> 4;
    return static_cast<uint64_t>((addr >> 4) & 0x3FFF) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFF) << 16) |
           (sbo << 32) | (1ull << 46) | (layout << 61);
}

/** Instruction descriptor of kind::f16 with both operands MN-major. */
__host__ __device__ constexpr uint32_t instr_desc_mn(int n) { return instr_desc(n) | (1u << 15) | (1u << 16); }

/** Weight gradient partials: for tap blockIdx.z, input channels ci0 =
 * 128 * (blockIdx.y / ntn) .. + 127 (rows past Cin are zero) and output
 * channels n0 = N * (blockIdx.y % ntn) .. + N - 1, the sum over the
 * pixel tiles t0 .. t1 - 1 of split blockIdx.x of X[p + off(tap)][ci] dY[p][co],
 * written (FP32, not accumulated) to part[((split * TAPS + tap) * cpad + ci) * Cout + co].
 * A = X shifted by the tap (M = input channels, K = 128 pixels per stage,
 * MN-major: atoms of KA channels), B = dY (N = output channels, MN-major:
 * atoms of KB channels); same roles of the warps as k_conv_tc. */
template <int TAPS, int KA, int KB>
__global__ void __launch_bounds__(kThreads, 1)
    k_conv_wgrad_tc(const __grid_constant__ CUtensorMap mapX, const __grid_constant__ CUtensorMap mapD,
                    float *__restrict__ part, int Cin, int Cout, int cpad, int N, int ntn, int Wt, int Ht,
                    int tiles_x, int tiles_y, int tiles_per_split, int ntiles, int S, uint32_t tmem_cols) {
    extern __shared__ __align__(1024) unsigned char conv_smem[];
    const uint32_t raw = smem_addr(conv_smem);
    const uint32_t base = (raw + 1023u) & ~1023u;
    constexpr uint32_t kAtomA = kTileM * KA * 2;  // one atom of KA channels for 128 pixels
    constexpr uint32_t abytes = (128 / KA) * kAtomA;
    const uint32_t atomB = kTileM * KB * 2, bbytes = (N / KB) * atomB;
    const uint32_t sA = base, sB = base + S * abytes;
    const uint32_t bar0 = sB + S * bbytes;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(conv_smem + (bar0 + 8 * (2 * S + 1) - raw));
    const uint32_t done = bar0 + 16 * S;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tap = blockIdx.z, ntile = blockIdx.y % ntn, ci0 = 128 * (blockIdx.y / ntn), n0 = N * ntile;
    const int dy = TAPS == 9 ? tap / 3 - 1 : 0, dx = TAPS == 9 ? tap % 3 - 1 : 0;
    const int t0 = blockIdx.x * tiles_per_split;
    const int t1 = t0 + tiles_per_split < ntiles ? t0 + tiles_per_split : ntiles;
    // channel atoms of A that hold input channels; the others stay zero
    const int natoms = ((Cin - ci0 < 128 ? Cin - ci0 : 128) + KA - 1) / KA;

    // zero the unused A atoms of every stage (generic proxy), then make the
    // stores visible to the tensor cores (async proxy)
    for (int s = 0; s < S; s++) {
        uint4 *za = reinterpret_cast<uint4 *>(conv_smem + (sA + s * abytes + natoms * kAtomA - raw));
        const int nz = static_cast<int>(((128 / KA) - natoms) * kAtomA / 16);
        for (int q = threadIdx.x; q < nz; q += blockDim.x) za[q] = make_uint4(0, 0, 0, 0);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (threadIdx.x == 0) {
        for (int q = 0; q < 2 * S + 1; q++) mbar_init(bar0 + 8 * q, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapX)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapD)) : "memory");
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int iters = t1 > t0 ? t1 - t0 : 0;

    if (threadIdx.x == 0) {
        int issued = 0;
        for (int it = 0; it < iters; it++) {
            const int s = it % S;
            if (it >= S && !mbar_wait(bar0 + 8 * (S + s), ((it / S) - 1) & 1)) break;
            int t = t0 + it;
            const int tx = t % tiles_x;
            t /= tiles_x;
            const int ty = t % tiles_y, b = t / tiles_y;
            const int x0 = tx * Wt, y0 = ty * Ht;
            const uint32_t full = bar0 + 8 * s;
            mbar_arrive_expect_tx(full, natoms * kAtomA + bbytes);
            for (int a = 0; a < natoms; a++)
                tma_load_4d(sA + s * abytes + a * kAtomA, &mapX, full, ci0 + a * KA, x0 + dx, y0 + dy, b);
            for (int a = 0; a < N / KB; a++)
                tma_load_4d(sB + s * bbytes + a * atomB, &mapD, full, n0 + a * KB, x0, y0, b);
            issued = it + 1;
        }
        for (int it = issued > S ? issued - S : 0; it < issued; it++) mbar_wait(bar0 + 8 * (it % S), (it / S) & 1);
    } else if (threadIdx.x == 32) {
        const uint32_t idesc = instr_desc_mn(N);
        for (int it = 0; it < iters; it++) {
            const int s = it % S;
            if (!mbar_wait(bar0 + 8 * s, (it / S) & 1)) break;
            tc_fence_after();
            const uint64_t ad = smem_desc_mn<KA>(sA + s * abytes, kAtomA);
            const uint64_t bd = smem_desc_mn<KB>(sB + s * bbytes, atomB);
            // K = 16 pixels per instruction: two swizzle groups of eight
            constexpr uint64_t stepA = (2 * 8 * 2 * KA) >> 4, stepB = (2 * 8 * 2 * KB) >> 4;
#pragma unroll
            for (int k = 0; k < kTileM / 16; k++)
                tc_mma(tmem, ad + stepA * k, bd + stepB * k, idesc, (it > 0 || k > 0) ? 1u : 0u);
            tc_commit(bar0 + 8 * (S + s));
        }
        tc_commit(done);
    }
    __syncwarp();

    bool ok = mbar_wait(done, 0);
    ok = __all_sync(0xffffffffu, ok);
    tc_fence_after();
    if (ok) {
        const int ci = ci0 + warp * 32 + lane;
        float *prow = part + ((static_cast<long>(blockIdx.x) * TAPS + tap) * cpad + ci) * Cout + n0;
        for (int c0 = 0; c0 < N; c0 += 16) {
            uint32_t v[16];
            tc_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0), v);
            if (ci >= Cin) continue;
            float4 *dst = reinterpret_cast<float4 *>(prow + c0);
#pragma unroll
            for (int j = 0; j < 4; j++)
                dst[j] = make_float4(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]),
                                     __uint_as_float(v[4 * j + 2]), __uint_as_float(v[4 * j + 3]));
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols) : "memory");
}

/** dW[tap][ci][co] += the splits' partials, summed in split order. */
__global__ void k_wgrad_reduce(const float *part, int splits, int taps, int Cin, int cpad, int Cout, float *dW) {
    const long n = static_cast<long>(taps) * Cin * Cout;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const int co = static_cast<int>(i % Cout);
        const long r = i / Cout;
        const int ci = static_cast<int>(r % Cin), tap = static_cast<int>(r / Cin);
        float acc = 0.f;
        for (int sp = 0; sp < splits; sp++)
            acc += part[((static_cast<long>(sp) * taps + tap) * cpad + ci) * Cout + co];
        dW[i] += acc;
    }
}

}  // namespace

namespace {

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

/** cuTensorMapEncodeTiled from the driver, through the runtime's entry-point
 * query (the library links the runtime only). */
EncodeTiled encode_tiled() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}

CUtensorMapSwizzle swizzle_of(int kc) {
    return kc == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : kc == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
}

constexpr int kMaxSmem = 227 * 1024;

template <int TAPS, int KC, bool ROWS, int HALVES = 1>
int launch_conv(const bf16 *X, int B, int H, int W, int Cin, const bf16 *wk, int Cout, int Nt, bool flip,
                const float *bias, bool relu, bf16 *Y, cudaStream_t s) {
    EncodeTiled enc = encode_tiled();
    if (!enc) {
        set_error("conv: cuTensorMapEncodeTiled is not available");
        return INCRMT_ERR_CUDA;
    }
    const int Wt = ROWS ? kRowsW : W >= 128 ? 128 : W >= 64 ? 64 : W >= 32 ? 32 : 16, Ht = HALVES * kTileM / Wt;
    const int tiles_x = (W + Wt - 1) / Wt, tiles_y = (H + Ht - 1) / Ht;
    CUtensorMap mA, mB;
    {
        const cuuint64_t dims[4] = {static_cast<cuuint64_t>(Cin), static_cast<cuuint64_t>(W),
                                    static_cast<cuuint64_t>(H), static_cast<cuuint64_t>(B)};
        const cuuint64_t strides[3] = {static_cast<cuuint64_t>(Cin) * 2, static_cast<cuuint64_t>(W) * Cin * 2,
                                       static_cast<cuuint64_t>(H) * W * Cin * 2};
        const cuuint32_t box[4] = {static_cast<cuuint32_t>(KC), static_cast<cuuint32_t>(Wt),
                                   static_cast<cuuint32_t>(ROWS ? Ht + 2 : Ht), 1};
        const cuuint32_t es[4] = {1, 1, 1, 1};
        CUresult r = enc(&mA, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(X), dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_of(KC), CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            set_error("conv: activation tensor map rejected (%d)", static_cast<int>(r));
            return INCRMT_ERR_CUDA;
        }
    }
    {
        const cuuint64_t dims[3] = {static_cast<cuuint64_t>(Cin), static_cast<cuuint64_t>(Cout),
                                    static_cast<cuuint64_t>(TAPS)};
        const cuuint64_t strides[2] = {static_cast<cuuint64_t>(Cin) * 2, static_cast<cuuint64_t>(Cout) * Cin * 2};
        const cuuint32_t box[3] = {static_cast<cuuint32_t>(KC), static_cast<cuuint32_t>(Nt), 1};
        const cuuint32_t es[3] = {1, 1, 1};
        CUresult r = enc(&mB, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<bf16 *>(wk), dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_of(KC), CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            set_error("conv: weight tensor map rejected (%d)", static_cast<int>(r));
            return INCRMT_ERR_CUDA;
        }
    }
    int S;
    size_t per;
    if (ROWS) {
        // as many stages as the CTA has steps, within a quarter of an SM's
        // shared memory (four CTAs per SM where the stages are small), at
        // least two
        per = static_cast<size_t>(HALVES * kTileM + 2 * kRowsW + 3 * Nt) * KC * 2;
        const int steps = 3 * (Cin / KC);
        S = static_cast<int>((56 * 1024) / per);
        if (S > steps) S = steps;
        if (S > 8) S = 8;
        if (S < 2) S = 2;
    } else {
        per = static_cast<size_t>(kTileM + Nt) * KC * 2;
        S = static_cast<int>((200 * 1024) / per);
        S = S > 4 ? 4 : S;
        if (S < 2) S = 2;
    }
    const size_t smem = 1024 + static_cast<size_t>(S) * per + 8 * (2 * S + 1) + 16;
    if (smem > static_cast<size_t>(kMaxSmem)) {
        set_error("conv: %zu bytes of shared memory needed", smem);
        return INCRMT_ERR_BADARG;
    }
    uint32_t cols = 32;
    while (cols < static_cast<uint32_t>(Nt)) cols <<= 1;
    cols *= HALVES;
    static bool attr = false;
    if (!attr) {
        INCRMT_CK(cudaFuncSetAttribute(k_conv_tc<TAPS, KC, ROWS, HALVES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kMaxSmem));
        attr = true;
    }
    const dim3 grid(static_cast<unsigned>(B * tiles_x * tiles_y), static_cast<unsigned>(Cout / Nt));
    k_conv_tc<TAPS, KC, ROWS, HALVES><<<grid, kThreads, smem, s>>>(mA, mB, bias, Y, H, W, Nt, Cout, Wt, Ht, tiles_x,
                                                                   tiles_y, Cin / KC, flip ? 1 : 0, relu ? 1 : 0, S,
                                                                   cols);
    INCRMT_CKL("k_conv_tc");
    return INCRMT_OK;
}

template <int TAPS, bool ROWS, int HALVES = 1>
int launch_taps(const bf16 *X, int B, int H, int W, int Cin, const bf16 *wk, int Cout, int Nt, bool flip,
                const float *bias, bool relu, bf16 *Y, cudaStream_t s) {
    if (Cin % 64 == 0)
        return launch_conv<TAPS, 64, ROWS, HALVES>(X, B, H, W, Cin, wk, Cout, Nt, flip, bias, relu, Y, s);
    if (Cin % 32 == 0)
        return launch_conv<TAPS, 32, ROWS, HALVES>(X, B, H, W, Cin, wk, Cout, Nt, flip, bias, relu, Y, s);
    return launch_conv<TAPS, 16, ROWS, HALVES>(X, B, H, W, Cin, wk, Cout, Nt, flip, bias, relu, Y, s);
}

/** Launch of k_conv_tc_persist; INCRMT_ERR_BADARG (nothing launched) when
 * the layer's weights and two stages do not fit in shared memory. */
template <int KC>
int launch_conv_persist(const bf16 *X, int B, int H, int W, int Cin, const bf16 *wk, int Cout, bool flip,
                        const float *bias, bool relu, bf16 *Y, cudaStream_t s) {
    EncodeTiled enc = encode_tiled();
    if (!enc) {
        set_error("conv: cuTensorMapEncodeTiled is not available");
        return INCRMT_ERR_CUDA;
    }
    const int nck = Cin / KC;
    const size_t abytes = static_cast<size_t>(kTileM + 2 * kRowsW) * KC * 2;
    const size_t wbytes = 9ull * nck * Cout * KC * 2;
    const size_t fixed = 1024 + wbytes + 8 * 6 + 16;
    if (fixed + 2 * (abytes + 16) > static_cast<size_t>(kMaxSmem)) {
        set_error("conv: weights of %zu bytes leave no room for two stages", wbytes);
        return INCRMT_ERR_BADARG;
    }
    int S = static_cast<int>((kMaxSmem - fixed) / (abytes + 16));
    if (S > 8) S = 8;
    const size_t smem = fixed + S * abytes + 16 * S;
    const int tiles_x = (W + kRowsW - 1) / kRowsW, tiles_y = (H + kRowsH - 1) / kRowsH;
    const int ntiles = B * tiles_x * tiles_y;
    CUtensorMap mA, mB;
    {
        const cuuint64_t dims[4] = {static_cast<cuuint64_t>(Cin), static_cast<cuuint64_t>(W),
                                    static_cast<cuuint64_t>(H), static_cast<cuuint64_t>(B)};
        const cuuint64_t strides[3] = {static_cast<cuuint64_t>(Cin) * 2, static_cast<cuuint64_t>(W) * Cin * 2,
                                       static_cast<cuuint64_t>(H) * W * Cin * 2};
        const cuuint32_t box[4] = {static_cast<cuuint32_t>(KC), static_cast<cuuint32_t>(kRowsW),
                                   static_cast<cuuint32_t>(kRowsH + 2), 1};
        const cuuint32_t es[4] = {1, 1, 1, 1};
        CUresult r = enc(&mA, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(X), dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_of(KC), CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            set_error("conv: activation tensor map rejected (%d)", static_cast<int>(r));
            return INCRMT_ERR_CUDA;
        }
    }
    {
        const cuuint64_t dims[3] = {static_cast<cuuint64_t>(Cin), static_cast<cuuint64_t>(Cout), 9};
        const cuuint64_t strides[2] = {static_cast<cuuint64_t>(Cin) * 2, static_cast<cuuint64_t>(Cout) * Cin * 2};
        const cuuint32_t box[3] = {static_cast<cuuint32_t>(KC), static_cast<cuuint32_t>(Cout), 1};
        const cuuint32_t es[3] = {1, 1, 1};
        CUresult r = enc(&mB, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<bf16 *>(wk), dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_of(KC), CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            set_error("conv: weight tensor map rejected (%d)", static_cast<int>(r));
            return INCRMT_ERR_CUDA;
        }
    }
    uint32_t cols = 32;
    while (cols < static_cast<uint32_t>(Cout)) cols <<= 1;
    static bool attr = false;
    if (!attr) {
        INCRMT_CK(cudaFuncSetAttribute(k_conv_tc_persist<KC>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem));
        attr = true;
    }
    int occ = 0;
    INCRMT_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_conv_tc_persist<KC>, kPersistThreads, smem));
    if (occ < 1) occ = 1;
    while (occ > 1 && occ * 2 * cols > 512) occ--;  // two accumulators per CTA in the SM's 512 columns
    const int grid = ntiles < kB200SMs * occ ? ntiles : kB200SMs * occ;
    k_conv_tc_persist<KC><<<grid, kPersistThreads, smem, s>>>(mA, mB, bias, Y, H, W, Cout, tiles_x, tiles_y, ntiles,
                                                              nck, flip ? 1 : 0, relu ? 1 : 0, S, cols);
    INCRMT_CKL("k_conv_tc_persist");
    return INCRMT_OK;
}

int g_conv_variant = 0;  // 0 automatic, 1 one tap per stage, 2 row reuse, 3 resident weights, 4 two halves

/** Split of the weight gradient over the pixels: about four waves of CTAs
 * over the SMs. */
struct WgradPlan {
    int Wt, Ht, tiles_x, tiles_y, ntiles, ci_tiles, cpad, Nt, ntn, tiles_per_split, splits;
};

WgradPlan wgrad_plan(int B, int H, int W, int Cin, int Cout, int taps) {
    WgradPlan p;
    p.Wt = W >= 128 ? 128 : W >= 64 ? 64 : W >= 32 ? 32 : 16;
    p.Ht = kTileM / p.Wt;
    p.tiles_x = (W + p.Wt - 1) / p.Wt;
    p.tiles_y = (H + p.Ht - 1) / p.Ht;
    p.ntiles = B * p.tiles_x * p.tiles_y;
    p.ci_tiles = (Cin + 127) / 128;
    p.cpad = 128 * p.ci_tiles;
    p.Nt = Cout;
    if (p.Nt > 256) {
        p.Nt = 256;
        while (Cout % p.Nt) p.Nt -= 16;
    }
    p.ntn = Cout / p.Nt;
    const int groups = taps * p.ci_tiles * p.ntn;
    int splits = (4 * kB200SMs + groups - 1) / groups;
    if (splits > p.ntiles) splits = p.ntiles;
    if (splits < 1) splits = 1;
    p.tiles_per_split = (p.ntiles + splits - 1) / splits;
    p.splits = (p.ntiles + p.tiles_per_split - 1) / p.tiles_per_split;  // every split has a tile
    return p;
}

template <int TAPS, int KA, int KB>
int launch_wgrad(const bf16 *X, const bf16 *dY, int B, int H, int W, int Cin, int Cout, float *dW, float *part,
                 const WgradPlan &p, cudaStream_t s) {
    EncodeTiled enc = encode_tiled();
    if (!enc) {
        set_error("conv: cuTensorMapEncodeTiled is not available");
        return INCRMT_ERR_CUDA;
    }
    CUtensorMap mX, mD;
    const cuuint32_t es[4] = {1, 1, 1, 1};
    auto encode = [&](CUtensorMap *m, const bf16 *ptr, int C, int box_c, CUtensorMapSwizzle sw) -> CUresult {
        const cuuint64_t dims[4] = {static_cast<cuuint64_t>(C), static_cast<cuuint64_t>(W), static_cast<cuuint64_t>(H),
                                    static_cast<cuuint64_t>(B)};
        const cuuint64_t strides[3] = {static_cast<cuuint64_t>(C) * 2, static_cast<cuuint64_t>(W) * C * 2,
                                       static_cast<cuuint64_t>(H) * W * C * 2};
        const cuuint32_t box[4] = {static_cast<cuuint32_t>(box_c), static_cast<cuuint32_t>(p.Wt),
                                   static_cast<cuuint32_t>(p.Ht), 1};
        return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(ptr), dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    };
    if (encode(&mX, X, Cin, KA, swizzle_of(KA)) != CUDA_SUCCESS || encode(&mD, dY, Cout, KB, swizzle_of(KB)) != CUDA_SUCCESS) {
        set_error("conv: weight-gradient tensor map rejected");
        return INCRMT_ERR_CUDA;
    }
    const int per = kTileM * 128 * 2 + p.Nt * kTileM * 2;
    int S = (200 * 1024) / per;
    S = S > 4 ? 4 : S;
    if (S < 2) S = 2;
    const size_t smem = 1024 + static_cast<size_t>(S) * per + 8 * (2 * S + 1) + 16;
    uint32_t cols = 32;
    while (cols < static_cast<uint32_t>(p.Nt)) cols <<= 1;
    static bool attr = false;
    if (!attr) {
        INCRMT_CK(cudaFuncSetAttribute(k_conv_wgrad_tc<TAPS, KA, KB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kMaxSmem));
        attr = true;
    }
    const dim3 grid(static_cast<unsigned>(p.splits), static_cast<unsigned>(p.ci_tiles * p.ntn), TAPS);
    k_conv_wgrad_tc<TAPS, KA, KB><<<grid, kThreads, smem, s>>>(mX, mD, part, Cin, Cout, p.cpad, p.Nt, p.ntn, p.Wt,
                                                               p.Ht, p.tiles_x, p.tiles_y, p.tiles_per_split,
                                                               p.ntiles, S, cols);
    INCRMT_CKL("k_conv_wgrad_tc");
    const long n = static_cast<long>(TAPS) * Cin * Cout;
    const long nb = (n + 255) / 256;
    k_wgrad_reduce<<<static_cast<unsigned>(nb < 4L * kB200SMs ? nb : 4L * kB200SMs), 256, 0, s>>>(
        part, p.splits, TAPS, Cin, p.cpad, Cout, dW);
    INCRMT_CKL("k_wgrad_reduce");
    return INCRMT_OK;
}

template <int TAPS, int KA>
int wgrad_kb(const bf16 *X, const bf16 *dY, int B, int H, int W, int Cin, int Cout, float *dW, float *part,
             const WgradPlan &p, cudaStream_t s) {
    if (p.Nt % 64 == 0) return launch_wgrad<TAPS, KA, 64>(X, dY, B, H, W, Cin, Cout, dW, part, p, s);
    if (p.Nt % 32 == 0) return launch_wgrad<TAPS, KA, 32>(X, dY, B, H, W, Cin, Cout, dW, part, p, s);
    return launch_wgrad<TAPS, KA, 16>(X, dY, B, H, W, Cin, Cout, dW, part, p, s);
}

template <int TAPS>
int wgrad_ka(const bf16 *X, const bf16 *dY, int B, int H, int W, int Cin, int Cout, float *dW, float *part,
             const WgradPlan &p, cudaStream_t s) {
    if (Cin % 64 == 0) return wgrad_kb<TAPS, 64>(X, dY, B, H, W, Cin, Cout, dW, part, p, s);
    if (Cin % 32 == 0) return wgrad_kb<TAPS, 32>(X, dY, B, H, W, Cin, Cout, dW, part, p, s);
    return wgrad_kb<TAPS, 16>(X, dY, B, H, W, Cin, Cout, dW, part, p, s);
}

}  // namespace

size_t conv_tc_wgrad_workspace(int B, int H, int W, int Cin, int Cout, int taps) {
    const WgradPlan p = wgrad_plan(B, H, W, Cin, Cout, taps);
    return static_cast<size_t>(p.splits) * taps * p.cpad * Cout;
}

int conv_tc_wgrad(const bf16 *X, const bf16 *dY, int B, int H, int W, int Cin, int Cout, int taps, float *dW,
                  float *part, size_t part_floats, cudaStream_t s) {
    if (!X || !dY || !dW || !part || B < 1 || H < 1 || W < 1 || Cin < 16 || Cin % 16 || Cout < 16 || Cout % 16 ||
        (taps != 1 && taps != 9)) {
        set_error("conv: bad weight-gradient arguments");
        return INCRMT_ERR_BADARG;
    }
    const WgradPlan p = wgrad_plan(B, H, W, Cin, Cout, taps);
    if (part_floats < static_cast<size_t>(p.splits) * taps * p.cpad * Cout) {
        set_error("conv: weight-gradient workspace too small");
        return INCRMT_ERR_BADARG;
    }
    if (taps == 9) return wgrad_ka<9>(X, dY, B, H, W, Cin, Cout, dW, part, p, s);
    return wgrad_ka<1>(X, dY, B, H, W, Cin, Cout, dW, part, p, s);
}

int conv_tc(const bf16 *X, int B, int H, int W, int Cin, const bf16 *wk, int taps, int Cout, bool flip,
            const float *bias, bool relu, bf16 *Y, cudaStream_t s) {
    if (!X || !wk || !Y || B < 1 || H < 1 || W < 1 || Cin < 16 || Cin % 16 || Cout < 16 || Cout % 16 ||
        (taps != 1 && taps != 9)) {
        set_error("conv: bad arguments (channels must be positive multiples of 16, taps 1 or 9)");
        return INCRMT_ERR_BADARG;
    }
    // Two 128-pixel halves per CTA (variant 4): the weights of each stage
    // serve 256 pixels. The default for up to 32 outputs, and for up to 64
    // from at most 32 inputs (2048^2, 32 -> 32: 384 against 291 TFLOP/s;
    // 1024^2, 32 -> 64: 379 against 336 with resident weights; 64 -> 64 is
    // faster with resident weights, 537 against 364).
    const bool halves = g_conv_variant == 4 || (g_conv_variant == 0 && (Cout <= 32 || (Cout <= 64 && Cin <= 32)));
    if (taps == 9 && halves && Cout <= 64)
        return launch_taps<9, true, 2>(X, B, H, W, Cin, wk, Cout, Cout, flip, bias, relu, Y, s);
    // Resident weights (persistent CTAs) where a 3x3 layer's weights take at
    // most 160 KB with 64 to 128 output channels, the default there. With
    // fewer outputs each tile's MMAs are too short for one CTA's four
    // epilogue warps to keep up, and row reuse with several CTAs per SM is
    // faster (2048^2, 32 -> 32: 291 against 186 TFLOP/s).
    if (taps == 9 && Cout <= 128 && 9ull * Cin * Cout * 2 <= 160 * 1024 &&
        (g_conv_variant == 3 || (g_conv_variant == 0 && Cout >= 64))) {
        if (Cin % 64 == 0) return launch_conv_persist<64>(X, B, H, W, Cin, wk, Cout, flip, bias, relu, Y, s);
        if (Cin % 32 == 0) return launch_conv_persist<32>(X, B, H, W, Cin, wk, Cout, flip, bias, relu, Y, s);
        return launch_conv_persist<16>(X, B, H, W, Cin, wk, Cout, flip, bias, relu, Y, s);
    }
    // Row reuse (3x3) for up to 128 output channels per CTA, where its three
    // taps' weights per stage still leave room for two CTAs per SM; one tap
    // per stage above that.
    const bool rows = taps == 9 && (g_conv_variant == 2 || (g_conv_variant != 1 && Cout <= 128));
    // output channels per CTA: all of them up to the cap (128 with row reuse,
    // else 256), else the largest multiple of 16 below the cap dividing Cout
    const int cap = rows ? 128 : 256;
    int Nt = Cout;
    if (Nt > cap) {
        Nt = cap;
        while (Cout % Nt) Nt -= 16;
    }
    if (rows) return launch_taps<9, true>(X, B, H, W, Cin, wk, Cout, Nt, flip, bias, relu, Y, s);
    if (taps == 9) return launch_taps<9, false>(X, B, H, W, Cin, wk, Cout, Nt, flip, bias, relu, Y, s);
    return launch_taps<1, false>(X, B, H, W, Cin, wk, Cout, Nt, flip, bias, relu, Y, s);
}

int conv_tc_set_variant(int v) {
    if (v < 0 || v > 4) {
        set_error("conv: variant %d not in 0..4", v);
        return INCRMT_ERR_BADARG;
    }
    g_conv_variant = v;
    return INCRMT_OK;
}

int conv_tc_status() {
    INCRMT_CK(cudaDeviceSynchronize());
    int flag = 0, zero = 0;
    INCRMT_CK(cudaMemcpyFromSymbol(&flag, g_conv_timeout, sizeof(int)));
    if (flag) {
        INCRMT_CK(cudaMemcpyToSymbol(g_conv_timeout, &zero, sizeof(int)));
        set_error("tensor-core convolution: a pipeline wait exceeded its one-second limit");
        return INCRMT_ERR_CUDA;
    }
    return INCRMT_OK;
}

}  // namespace incrmt
