// unet_conv.cu — 3x3x3 convolution as an implicit GEMM on the tcgen05
// tensor cores (BF16 operands, FP32 accumulation in tensor memory).
//
// Activations are channels-last with a one-voxel zero halo on every side:
// element (x, y, z, c) of a W x H x D x C tensor sits at
// ((z+1)*Hp + (y+1))*Wp + (x+1)) * C + c with Wp = W+2, Hp = H+2, plus
// kSlack zero voxels before and after the tensor.  Weights are [27][Cout][Cin]
// (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)), bias FP32 [Cout].
//
// One CTA computes M = 128 consecutive voxels of the padded plane z (its
// interior rows) for all N = Cout outputs.  For each 16-channel chunk of the
// input it stages the 9 input rows (dy, dz) of 130 voxels once, in the
// canonical K-major layout of the UMMA operand descriptor (8-voxel core
// matrices of 16 B rows, 128 B apart; the two 8-channel halves 2080 B
// apart).  Because a voxel's row is exactly 16 B at a linear position, the
// A operand of tap (dx, dy, dz) is the same block seen 16*(dx+1) B further
// on: 27 MMAs of M=128 x N x K=16 read one staged block.  The halo makes
// the zero padding of the convolution a plain memory read.
#include <cuda_bf16.h>

#include "kernels.cuh"

namespace blz {

namespace {

constexpr int kConvM = 128;
constexpr int kRowVox = kConvM + 2;                 // 130 voxels per staged row
constexpr int kKgBytes = kRowVox * 16;              // one 8-channel half of a row
constexpr int kRowBytes = 2 * kKgBytes;             // 4160 B per staged row (16 ch)
constexpr int kABytes = 9 * kRowBytes;              // 37440 B

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor: K-major, no swizzle (canonical layout
// ((8,m),2):((1,SBO),LBO) in 16-byte units), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;                          // version
    return d;                                        // base offset 0, layout SWIZZLE_NONE
}

// Instruction descriptor, kind::f16: D FP32, A and B BF16, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

__device__ __forceinline__ void st_shared_zero16(uint32_t dst) {
    asm volatile("st.shared.v4.u32 [%0], {%1, %1, %1, %1};" ::"r"(dst), "r"(0u) : "memory");
}

__device__ __forceinline__ unsigned long long conv_now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// A commit group of one tile's MMAs completes in microseconds.
constexpr unsigned long long kConvWaitNs = 10ull * 1000ull * 1000ull;

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, int *err) {
    // Bounded in time (device global timer): gives up after kConvWaitNs,
    // records the timeout and returns.
    const unsigned long long t0 = conv_now_ns();
    for (;;) {
        for (int it = 0; it < 64; ++it) {
            uint32_t done;
            asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                         " selp.u32 %0, 1, 0, p;\n}\n"
                         : "=r"(done) : "r"(mbar), "r"(parity) : "memory");
            if (done) return true;
        }
        if (conv_now_ns() - t0 > kConvWaitNs) break;
    }
    if (err) atomicExch(err, 1);
    return false;
}

} // namespace

template <int N, bool RELU, bool OUT_F32>
__global__ void __launch_bounds__(128, 1)
k_conv3d_tc(int W, int H, int D, int cin, int out_stride, int out_offset, const __nv_bfloat16 *__restrict__ x,
            const __nv_bfloat16 *__restrict__ w, const float *__restrict__ bias, void *__restrict__ y,
            const __nv_bfloat16 *__restrict__ aux, int *err) {
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *sA = smem;
    unsigned char *sB = smem + kABytes;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    constexpr int kCols = N < 32 ? 32 : N;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Wp = W + 2, Hp = H + 2;
    const long long plane = (long long)Wp * Hp;
    const int z = blockIdx.y;
    const long long P0 = (long long)Wp + (long long)kConvM * blockIdx.x;   // first voxel of the tile

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base)), "r"(kCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    const uint32_t aS = smem_u32(sA), bS = smem_u32(sB), mb = smem_u32(&mbar);
    constexpr uint32_t idesc = umma_idesc_bf16(kConvM, N);
    const int chunks = cin / 16;
    bool ok = true;
    for (int c = 0; c < chunks && ok; ++c) {
        // Stage the 9 input rows (dz, dy) of this 16-channel chunk: row r =
        // (dz + 1) * 3 + (dy + 1) holds 16-byte chunks (kg, v) at kg *
        // kKgBytes + v * 16, from voxel v of that row ...
#pragma unroll
        for (int r = 0; r < 9; ++r) {
            const int dz = r / 3 - 1, dy = r % 3 - 1;
            const __nv_bfloat16 *rs =
                x + ((long long)(z + 1 + dz) * plane + P0 - 1 + (long long)dy * Wp) * cin + c * 16;
            for (int e = tid; e < 2 * kRowVox; e += 128) {
                const int kg = e & 1, v = e >> 1;
                cp_async16(aS + r * kRowBytes + kg * kKgBytes + v * 16, rs + (long long)v * cin + kg * 8);
            }
        }
        // ... and the 27 taps' weights of the chunk (B: N x 16, K-major).
        for (int e = tid; e < 27 * N * 2; e += 128) {
            const int t = e / (N * 2), rem = e % (N * 2);
            const int n = rem >> 1, kg = rem & 1;
            cp_async16(bS + t * N * 32 + kg * N * 16 + n * 16, w + ((size_t)t * N + n) * cin + c * 16 + kg * 8);
        }
        asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // a tap's operands: the block's descriptors plus constant offsets
            // in the 16-byte address field (addresses below 2^18 bytes, so
            // the field never carries)
            const uint64_t a_desc0 = umma_desc(aS, kKgBytes, 128), b_desc0 = umma_desc(bS, N * 16, 128);
#pragma unroll
            for (int t = 0; t < 27; ++t) {
                const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
                const int r = (dz + 1) * 3 + (dy + 1);
                const uint64_t ad = a_desc0 + (uint64_t)((r * kRowBytes + (dx + 1) * 16) >> 4);
                const uint64_t bd = b_desc0 + (uint64_t)((t * N * 32) >> 4);
                const uint32_t acc = (c > 0 || t > 0) ? 1u : 0u;
                asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                             " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                             ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(mb) : "memory");
        }
        // The staged block is reused by the next chunk only once the MMAs
        // that read it have completed.
        // (CTA-uniform outcome, so the .sync.aligned TMEM loads below never
        // run in a divergent warp.)
        ok = __syncthreads_and(mbar_wait(mb, (uint32_t)(c & 1), err)) != 0;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
        // Epilogue: warp w owns TMEM lanes 32w..32w+31 = voxels of the tile.
        const long long P = P0 + 32 * warp + lane;
        const int xp = (int)(P % Wp), yp = (int)(P / Wp);
        const bool inside = xp >= 1 && xp <= W && yp >= 1 && yp <= H;
        const long long outv = (long long)(z + 1) * plane + P;
#pragma unroll
        for (int n0 = 0; n0 < N; n0 += 16) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)n0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
                           "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                         : "r"(taddr) : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (inside) {
                float v[16];
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    v[q] = __uint_as_float(r[q]) + (bias ? __ldg(bias + n0 + q) : 0.0f);
                    if (RELU) v[q] = fmaxf(v[q], 0.0f);
                }
                const long long o = outv * out_stride + out_offset + n0;
                if (aux) {
                    // Backward through a ReLU: keep the gradient where the
                    // forward activation was positive.
                    const uint4 a0 = __ldg(reinterpret_cast<const uint4 *>(aux + o));
                    const uint4 a1 = __ldg(reinterpret_cast<const uint4 *>(aux + o) + 1);
                    const __nv_bfloat16 *ah0 = reinterpret_cast<const __nv_bfloat16 *>(&a0);
                    const __nv_bfloat16 *ah1 = reinterpret_cast<const __nv_bfloat16 *>(&a1);
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        if (!(__bfloat162float(ah0[q]) > 0.0f)) v[q] = 0.0f;
                        if (!(__bfloat162float(ah1[q]) > 0.0f)) v[8 + q] = 0.0f;
                    }
                }
                if (OUT_F32) {
                    float4 *dst = reinterpret_cast<float4 *>(static_cast<float *>(y) + o);
#pragma unroll
                    for (int q = 0; q < 4; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                } else {
                    __nv_bfloat162 h[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) h[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
                    uint4 *dst = reinterpret_cast<uint4 *>(static_cast<__nv_bfloat16 *>(y) + o);
                    dst[0] = *reinterpret_cast<uint4 *>(&h[0]);
                    dst[1] = *reinterpret_cast<uint4 *>(&h[4]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

int conv3d_smem_bytes(int cout) { return kABytes + 27 * cout * 32; }

// ---------------------------------------------------------------------------
// z-marching variant for layers with cin, cout in {16, 32} (the full- and
// half-resolution layers, which carry most of the network's voxels).  A CTA
// keeps the layer's weights resident in shared memory and walks one 128-voxel
// tile through `zs` consecutive planes.  Output plane z needs input planes
// z-1, z, z+1 (padded planes z, z+1, z+2), 3 rows each.  They arrive by TMA
// (one tensor-map box per row, completing on the slot's mbarrier by
// transaction count) in a ring of S plane slots, S - 2 planes ahead, so each
// plane's rows are staged once per tile and their latency is hidden behind
// several planes; the TMEM accumulator has kZmAcc buffers.  The CTA is warp
// specialised and its warps hand over through mbarriers only:
//   workers (warps 0-3), iteration z: thread 0 issues the copies of padded
//   plane z+S-2 (into the slot of plane z-2, whose last reader, plane z-2's
//   MMAs, completed before the workers read that plane out) | all wait for
//   plane z-1's MMAs (accf), read its accumulator from TMEM, add bias /
//   ReLU, store, arrive on acce (buffer free);
//   MMA warp (warp 4), iteration z: wait full[] of plane z+2 and acce of
//   buffer z % kZmAcc (read out by iteration z-kZmAcc) | lane 0 issues
//   27 x cin/16 MMAs into that buffer and commits to its accf.
// So the MMA warp runs up to kZmAcc - 1 planes ahead of the workers.  Every
// wait is bounded in time; a wait that gives up sets the error flag and ends
// that warp's loop, which ends the others' at their next (bounded) wait;
// before the CTA ends, the MMA warp waits for its last commit and thread 0
// for the latest copy into every slot.
// S is as many slots as fit, at most 8: with two CTAs per SM when at least 6
// fit in half the SM's shared memory (two independent pipelines), else with
// one CTA.
// ---------------------------------------------------------------------------
constexpr int kZmWorkers = 128;                           // staging + epilogue warps 0-3
constexpr int kZmThreads = kZmWorkers + 32;               // + the MMA warp
constexpr int kZmAcc = 4;                                 // accumulator buffers in TMEM
constexpr int kZmSmemOne = 227 * 1024 - 1024;            // dynamic bytes, one CTA per SM
constexpr int kZmSmemTwo = 228 * 1024 / 2 - 1024 - 128;  // dynamic bytes, two CTAs per SM

// A slot holds the rows dy = -1, 0, 1 of one padded plane, each row block
// [ch][kg][v][8 channels] (CIN/16 chunks of two 8-channel halves of 130
// voxels) as one TMA box, the blocks 128-byte aligned.
template <int CIN> __host__ __device__ constexpr int zm_dy_bytes() { return ((CIN / 16) * kRowBytes + 127) & ~127; }
template <int CIN> __host__ __device__ constexpr int zm_slot_bytes() { return 3 * zm_dy_bytes<CIN>(); }
template <int N, int CIN> __host__ __device__ constexpr int zm_w_bytes() { return 27 * (CIN / 16) * N * 32; }
// dynamic shared memory besides the slots: the weights and 128 bytes of
// alignment slack
template <int N, int CIN> __host__ __device__ constexpr int zm_fixed_bytes() { return zm_w_bytes<N, CIN>() + 128; }
template <int N, int CIN> __host__ __device__ constexpr int zm_slots() {
    return (kZmSmemTwo - zm_fixed_bytes<N, CIN>()) / zm_slot_bytes<CIN>() >= 6
               ? ((kZmSmemTwo - zm_fixed_bytes<N, CIN>()) / zm_slot_bytes<CIN>() > 8
                      ? 8 : (kZmSmemTwo - zm_fixed_bytes<N, CIN>()) / zm_slot_bytes<CIN>())
               : ((kZmSmemOne - zm_fixed_bytes<N, CIN>()) / zm_slot_bytes<CIN>() > 8
                      ? 8 : (kZmSmemOne - zm_fixed_bytes<N, CIN>()) / zm_slot_bytes<CIN>());
}
template <int N, int CIN> __host__ __device__ constexpr int zm_smem_bytes() {
    return zm_fixed_bytes<N, CIN>() + zm_slots<N, CIN>() * zm_slot_bytes<CIN>();
}
static_assert(zm_w_bytes<16, 16>() % 128 == 0 && zm_w_bytes<32, 32>() % 128 == 0 && zm_dy_bytes<16>() == 4224 &&
                  zm_dy_bytes<32>() == 8320, "128-byte aligned slots");
static_assert(zm_slots<16, 16>() == 8 && zm_slots<32, 16>() == 6 && zm_slots<16, 32>() == 8 &&
                  zm_slots<32, 32>() == 7, "ring slots of the z-marching convolution");
static_assert(zm_smem_bytes<16, 16>() <= kZmSmemTwo && zm_smem_bytes<32, 16>() <= kZmSmemTwo &&
                  zm_smem_bytes<16, 32>() <= kZmSmemOne && zm_smem_bytes<32, 32>() <= kZmSmemOne,
              "shared memory of the z-marching convolution");

template <int N, int CIN, bool RELU>
__global__ void __launch_bounds__(kZmThreads, 1)
k_conv3d_zm(int W, int H, int D, int zs, int out_stride, int out_offset, const __grid_constant__ CUtensorMap xmap,
            const __nv_bfloat16 *__restrict__ w, const float *__restrict__ bias, __nv_bfloat16 *__restrict__ y,
            const __nv_bfloat16 *__restrict__ aux, int *err) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int CH = CIN / 16;
    constexpr int S = zm_slots<N, CIN>();
    constexpr int kSlot = zm_slot_bytes<CIN>();
    constexpr int kDy = zm_dy_bytes<CIN>();
    constexpr uint32_t kSlotTx = 3u * CH * kRowBytes;       // bytes the three row boxes of a plane bring
    constexpr int kCols = kZmAcc * N < 32 ? 32 : kZmAcc * N;   // a power of two
    constexpr uint32_t idesc = umma_idesc_bf16(kConvM, N);
    // full[s]: the plane in ring slot s has landed (the TMA copies' bytes);
    // accf[b]: the MMAs into accumulator buffer b completed (their commit);
    // acce[b]: buffer b has been read out (one arrival per worker).  Plane
    // iteration it uses buffer it % kZmAcc, the n-th time for n = it / kZmAcc.
    __shared__ __align__(8) uint64_t full[S], accf[kZmAcc], acce[kZmAcc];
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool worker = warp < 4;
    const int Wp = W + 2, Hp = H + 2;
    const long long plane = (long long)Wp * Hp;
    const long long P0 = (long long)Wp + (long long)kConvM * blockIdx.x;
    const int z0 = blockIdx.y * zs;
    const int nz = (z0 + zs < D ? z0 + zs : D) - z0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base)), "r"(kCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < S; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[s])) : "memory");
        for (int b = 0; b < kZmAcc; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&accf[b])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&acce[b])), "r"(kZmWorkers) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    const uint32_t bS = (smem_u32(smem) + 127u) & ~127u;       // weights, then the ring, 128-byte aligned
    const uint32_t aS = bS + (uint32_t)zm_w_bytes<N, CIN>();
    // Ring slot of padded plane pz: (pz - z0) % S, so the n-th fill of a slot
    // is the plane z0 + s + n S and completes phase n of full[s].
    auto slot_of = [&](int pz) { return (pz - z0) % S; };
    auto fill_parity = [&](int pz) { return (uint32_t)(((pz - z0) / S) & 1); };
    // Weights of every 16-channel chunk: block (ch, tap) = N rows x 32 B,
    // K-major (cp.async by the workers, fenced to the async proxy before the
    // barrier that starts the pipeline).
    if (worker) {
        for (int e = tid; e < 27 * CH * N * 2; e += kZmWorkers) {
            const int kg = e & 1, n = (e >> 1) % N, ct = (e >> 1) / N;      // ct = ch * 27 + tap
            const int ch = ct / 27, t = ct % 27;
            cp_async16(bS + ct * N * 32 + kg * N * 16 + n * 16, w + ((size_t)t * N + n) * CIN + ch * 16 + kg * 8);
        }
        asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    // Padded plane pz by TMA: rows dy = -1, 0, 1 of the tile (130 voxels
    // each: its 128 and one either side, flattened in-plane index P0 - 1 +
    // (dy - 1) Wp on), one box per row of 8 channels x 130 voxels x 2
    // halves x 1 plane x CIN/16 chunks, landing as [ch][kg][v][8] at
    // dy * kDy in the slot; voxels outside the plane read as zeros.
    auto tma_plane = [&](int pz) {
        const uint32_t bar = smem_u32(&full[slot_of(pz)]);
        const uint32_t dst = aS + (uint32_t)(slot_of(pz) * kSlot);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kSlotTx) : "memory");
#pragma unroll
        for (int dy = 0; dy < 3; ++dy)
            asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                         " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
                         ::"r"(dst + (uint32_t)(dy * kDy)), "l"(reinterpret_cast<uint64_t>(&xmap)), "r"(0),
                           "r"((int)(P0 - 1) + (dy - 1) * Wp), "r"(0), "r"(pz), "r"(0), "r"(bar)
                         : "memory");
    };
    int last_plane = z0 - 1;                             // last plane thread 0 asked for

    if (worker) {
        // ---- workers: thread 0 issues the plane copies; all drain the
        // accumulators ----
        // This thread's voxel of the tile (TMEM lane 32 * warp + lane) and
        // the bias, the same on every plane.
        const long long Pv = P0 + 32 * warp + lane;
        const int yv = (int)(Pv / Wp), xv = (int)(Pv - (long long)yv * Wp);
        const bool inside = xv >= 1 && xv <= W && yv >= 1 && yv <= H;
        float bv[N];
#pragma unroll
        for (int q = 0; q < N; ++q) bv[q] = bias ? __ldg(bias + q) : 0.0f;
        // Reads accumulator buffer it % kZmAcc (output plane z0 + it) and stores
        // it; false (the whole warp alike) when its wait gave up.
        auto epilogue = [&](int it) -> bool {
            const bool done = mbar_wait(smem_u32(&accf[it % kZmAcc]), (uint32_t)((it / kZmAcc) & 1), err);
            if (!__all_sync(0xffffffffu, done)) return false;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const long long outv = (long long)(z0 + it + 1) * plane + Pv;
#pragma unroll
            for (int n0 = 0; n0 < N; n0 += 16) {
                uint32_t r[16];
                const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)((it % kZmAcc) * N + n0);
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                               "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
                               "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                             : "r"(taddr) : "memory");
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (inside) {
                    float v[16];
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        v[q] = __uint_as_float(r[q]) + bv[n0 + q];
                        if (RELU) v[q] = fmaxf(v[q], 0.0f);
                    }
                    const long long o = outv * out_stride + out_offset + n0;
                    if (aux) {
                        const uint4 a0 = __ldg(reinterpret_cast<const uint4 *>(aux + o));
                        const uint4 a1 = __ldg(reinterpret_cast<const uint4 *>(aux + o) + 1);
                        const __nv_bfloat16 *ah0 = reinterpret_cast<const __nv_bfloat16 *>(&a0);
                        const __nv_bfloat16 *ah1 = reinterpret_cast<const __nv_bfloat16 *>(&a1);
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            if (!(__bfloat162float(ah0[q]) > 0.0f)) v[q] = 0.0f;
                            if (!(__bfloat162float(ah1[q]) > 0.0f)) v[8 + q] = 0.0f;
                        }
                    }
                    __nv_bfloat162 h[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) h[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
                    uint4 *dst = reinterpret_cast<uint4 *>(y + o);
                    dst[0] = *reinterpret_cast<uint4 *>(&h[0]);
                    dst[1] = *reinterpret_cast<uint4 *>(&h[4]);
                }
            }
            // the buffer may be overwritten by the MMAs of iteration it + kZmAcc
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acce[it % kZmAcc])) : "memory");
            return true;
        };
        // Prologue: padded planes z0 .. z0+S-3 (those the tile needs).
        if (tid == 0)
            for (int p = 0; p < S - 2 && p < nz + 2; ++p) {
                tma_plane(z0 + p);
                last_plane = z0 + p;
            }
        bool ok = true;
#pragma unroll 1
        for (int it = 0; it < nz && ok; ++it) {
            const int z = z0 + it;
            // plane z+S-2 goes into the slot of plane z-2, whose last reader
            // (the MMAs of iteration it-2) completed before this thread's
            // epilogue(it-2) returned
            if (tid == 0 && it + S - 2 < nz + 2) {
                tma_plane(z + S - 2);
                last_plane = z + S - 2;
            }
            if (it > 0) ok = epilogue(it - 1);
        }
        if (ok && nz > 0) ok = epilogue(nz - 1);
        if (!ok && err) atomicExch(err, 1);
        // No copy may land after the CTA ends: thread 0 waits (bounded) for
        // the latest fill of every slot it issued (done already unless a
        // wait gave up).
        if (tid == 0)
            for (int p = last_plane; p >= z0 && p > last_plane - S; --p)
                mbar_wait(smem_u32(&full[slot_of(p)]), fill_parity(p), nullptr);
    } else {
        // ---- MMA warp: lane 0 issues each plane's 27 x cin/16 MMAs ----
        // Operand descriptors at the start of the plane ring and of the
        // weights.  Every operand address stays below 2^18 bytes, so adding an
        // offset's 16-byte units to the 14-bit address field never carries.
        const uint64_t a_desc0 = umma_desc(aS, kKgBytes, 128);
        const uint64_t b_desc0 = umma_desc(bS, N * 16, 128);
        int issued = 0;
        bool ok = true;
#pragma unroll 1
        for (int it = 0; it < nz && ok; ++it) {
            const int z = z0 + it;
            bool done = true;
            if (it == 0) {
                done = mbar_wait(smem_u32(&full[slot_of(z)]), fill_parity(z), err) && done;
                done = mbar_wait(smem_u32(&full[slot_of(z + 1)]), fill_parity(z + 1), err) && done;
            }
            done = mbar_wait(smem_u32(&full[slot_of(z + 2)]), fill_parity(z + 2), err) && done;
            // accumulator buffer it % kZmAcc was last read out by epilogue(it - kZmAcc)
            if (it >= kZmAcc)
                done = mbar_wait(smem_u32(&acce[it % kZmAcc]), (uint32_t)(((it - kZmAcc) / kZmAcc) & 1), err) && done;
            if (!__all_sync(0xffffffffu, done)) { ok = false; break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (lane == 0) {
                const uint32_t acc = tmem + (uint32_t)((it % kZmAcc) * N);
                // descriptors of the slots of padded planes z, z+1, z+2 (taps
                // dz = -1, 0, +1); a tap's operand is its slot's descriptor
                // plus a constant offset in the 16-byte address field
                const uint64_t sz[3] = {a_desc0 + (uint64_t)((slot_of(z) * kSlot) >> 4),
                                        a_desc0 + (uint64_t)((slot_of(z + 1) * kSlot) >> 4),
                                        a_desc0 + (uint64_t)((slot_of(z + 2) * kSlot) >> 4)};
#pragma unroll
                for (int ch = 0; ch < CH; ++ch) {
#pragma unroll
                    for (int t = 0; t < 27; ++t) {
                        const int dzi = t / 9, dyi = (t / 3) % 3, dxi = t % 3;
                        const uint64_t ad = sz[dzi] + (uint64_t)((dyi * kDy + ch * kRowBytes + dxi * 16) >> 4);
                        const uint64_t bd = b_desc0 + (uint64_t)(((ch * 27 + t) * N * 32) >> 4);
                        const uint32_t accum = (ch > 0 || t > 0) ? 1u : 0u;
                        asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                                     " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                                     ::"r"(acc), "l"(ad), "l"(bd), "r"(idesc), "r"(accum) : "memory");
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             ::"r"(smem_u32(&accf[it % kZmAcc])) : "memory");
            }
            __syncwarp();
            issued = it + 1;
        }
        // The last committed MMAs complete before the accumulator columns are
        // released, also when a worker's wait gave up (bounded wait).
        if (issued > 0)
            mbar_wait(smem_u32(&accf[(issued - 1) % kZmAcc]), (uint32_t)(((issued - 1) / kZmAcc) & 1), nullptr);
        (void)ok;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

constexpr int kZmPlanes = 16;

// Tensor map of a padded channels-last activation x (CIN channels, W+2 x
// H+2 x D+2 voxels from x) for the z-marching convolution's row boxes:
// dims (8 channels, in-plane voxel, 8-channel half, plane, 16-channel chunk)
// with byte strides (2 CIN, 16, plane, 32), box (8, 130, 2, 1, CIN/16).  The
// innermost coordinate of every copy is 0, so every copy starts 16-byte
// aligned.
static bool zm_tensor_map(CUtensorMap *m, const __nv_bfloat16 *x, const ConvDesc &cd) {
    TensorMapEncodeFn enc = tensor_map_encoder();
    if (!enc || (reinterpret_cast<uintptr_t>(x) & 15) != 0) return false;
    const cuuint64_t Wp = (cuuint64_t)cd.W + 2, Hp = (cuuint64_t)cd.H + 2, Dp = (cuuint64_t)cd.D + 2;
    const cuuint64_t C = (cuuint64_t)cd.cin;
    const cuuint64_t dims[5] = {8, Wp * Hp, 2, Dp, C / 16};
    const cuuint64_t strides[4] = {C * 2, 16, Wp * Hp * C * 2, 32};
    const cuuint32_t box[5] = {8, (cuuint32_t)kRowVox, 2, 1, (cuuint32_t)(C / 16)};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16 *>(x), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int N, int CIN, bool RELU>
static cudaError_t launch_zm(const ConvDesc &cd, const __nv_bfloat16 *x, const __nv_bfloat16 *w, const float *bias,
                             void *y, const __nv_bfloat16 *aux, int *err, cudaStream_t st) {
    constexpr int smem = zm_smem_bytes<N, CIN>();
    cudaError_t e = cudaFuncSetAttribute(k_conv3d_zm<N, CIN, RELU>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    CUtensorMap xm;
    if (!zm_tensor_map(&xm, x, cd)) return cudaErrorNotSupported;
    const long long interior = (long long)(cd.W + 2) * cd.H;
    const dim3 grid((unsigned)((interior + kConvM - 1) / kConvM), (unsigned)((cd.D + kZmPlanes - 1) / kZmPlanes));
    const int os = cd.out_stride > 0 ? cd.out_stride : cd.cout;
    k_conv3d_zm<N, CIN, RELU><<<grid, kZmThreads, smem, st>>>(cd.W, cd.H, cd.D, kZmPlanes, os, cd.out_offset, xm, w, bias,
                                                       static_cast<__nv_bfloat16 *>(y), aux, err);
    return cudaGetLastError();
}

// The z-marching kernel for cin, cout in {16, 32} and BF16 output.
static bool zm_dispatch(const ConvDesc &cd, const __nv_bfloat16 *x, const __nv_bfloat16 *w, const float *bias,
                        void *y, const __nv_bfloat16 *aux, int *err, cudaStream_t st, cudaError_t *res) {
    if (cd.out_f32 || (cd.cin != 16 && cd.cin != 32) || (cd.cout != 16 && cd.cout != 32)) return false;
#define BLZ_ZM(NN, CC)                                                                              \
    if (cd.cout == NN && cd.cin == CC) {                                                            \
        *res = cd.relu ? launch_zm<NN, CC, true>(cd, x, w, bias, y, aux, err, st)                   \
                       : launch_zm<NN, CC, false>(cd, x, w, bias, y, aux, err, st);                 \
        return true;                                                                                \
    }
    BLZ_ZM(16, 16)
    BLZ_ZM(16, 32)
    BLZ_ZM(32, 16)
    BLZ_ZM(32, 32)
#undef BLZ_ZM
    return false;
}

template <int N, bool RELU, bool F32>
static cudaError_t launch_n(const ConvDesc &cd, const __nv_bfloat16 *x, const __nv_bfloat16 *w, const float *bias,
                            void *y, const __nv_bfloat16 *aux, int *err, cudaStream_t st) {
    const int smem = conv3d_smem_bytes(N);
    cudaError_t e = cudaFuncSetAttribute(k_conv3d_tc<N, RELU, F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const long long interior = (long long)(cd.W + 2) * cd.H;
    const dim3 grid((unsigned)((interior + kConvM - 1) / kConvM), (unsigned)cd.D);
    const int os = cd.out_stride > 0 ? cd.out_stride : cd.cout;
    k_conv3d_tc<N, RELU, F32><<<grid, 128, smem, st>>>(cd.W, cd.H, cd.D, cd.cin, os, cd.out_offset, x, w, bias, y,
                                                        aux, err);
    return cudaGetLastError();
}

cudaError_t launch_conv3d(const ConvDesc &cd, const __nv_bfloat16 *x, const __nv_bfloat16 *w, const float *bias,
                          void *y, int *err, cudaStream_t st, const __nv_bfloat16 *aux) {
    if (cd.cin % 16 || cd.cin <= 0 || cd.out_offset % 8 || (cd.out_stride > 0 && cd.out_stride % 8) ||
        (aux && cd.out_f32))
        return cudaErrorInvalidValue;
    cudaError_t res = cudaSuccess;
    if (zm_dispatch(cd, x, w, bias, y, aux, err, st, &res)) return res;
#define BLZ_CONV_CASE(NN)                                                                        \
    if (cd.cout == NN) {                                                                         \
        if (cd.out_f32) return cd.relu ? launch_n<NN, true, true>(cd, x, w, bias, y, aux, err, st) \
                                       : launch_n<NN, false, true>(cd, x, w, bias, y, aux, err, st); \
        return cd.relu ? launch_n<NN, true, false>(cd, x, w, bias, y, aux, err, st)             \
                       : launch_n<NN, false, false>(cd, x, w, bias, y, aux, err, st);          \
    }
    BLZ_CONV_CASE(16)
    BLZ_CONV_CASE(32)
    BLZ_CONV_CASE(64)
    BLZ_CONV_CASE(128)
#undef BLZ_CONV_CASE
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// 2x2x2 stride-2 transposed convolution on the tensor cores.  Fine voxel
// (2x+a, 2y+b, 2z+c) = bias + W[a + 2b + 4c] . x[x, y, z], so the 8 parities
// of a coarse voxel are one GEMM row: one CTA takes M = 128 consecutive
// padded coarse voxels of interior plane z (its interior rows, as the 3x3x3
// kernels tile a plane) and computes D[128 x 8 COUT] = X[128 x CIN] W^T with
// W in BF16 [8][COUT][CIN] (GEMM row n = par * COUT + co), K = 16 per MMA,
// N = 8 COUT split into MMAs of at most 256 columns.  Operands are staged
// once by cp.async in the canonical K-major layouts of the 3x3x3 kernels
// (A: [chunk][kg][voxel][8], B: [chunk][kg][n][8]); one thread issues the
// MMAs and commits them to an mbarrier (bounded wait); the epilogue reads
// each parity's COUT columns from TMEM, adds the bias and stores BF16 into
// the fine voxel's channels [0, COUT) of a tensor with channel stride ys.
// ---------------------------------------------------------------------------
template <int CIN, int COUT>
__global__ void __launch_bounds__(128, 1)
k_upconv_tc(int W, int H, int D, const __nv_bfloat16 *__restrict__ x, const __nv_bfloat16 *__restrict__ w,
            const float *__restrict__ bias, __nv_bfloat16 *__restrict__ y, int ys, int *err) {
    constexpr int N = 8 * COUT, CH = CIN / 16;
    constexpr int NMMA = N > 256 ? 256 : N;              // columns per MMA
    constexpr int kCols = N;                              // 128, 256 or 512: a power of two
    constexpr int kAChunk = 2 * kConvM * 16;              // [kg][voxel][8] of one 16-channel chunk
    constexpr int kBChunk = 2 * N * 16;                   // [kg][n][8] of one 16-channel chunk
    constexpr uint32_t idesc = umma_idesc_bf16(kConvM, NMMA);
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Wp = W + 2, Hp = H + 2;
    const long long plane = (long long)Wp * Hp;
    const int z = blockIdx.y;                                              // interior coarse plane
    const long long P0 = (long long)Wp + (long long)kConvM * blockIdx.x;   // first voxel of the tile

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base)), "r"(kCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    const uint32_t aS = smem_u32(smem), bS = aS + (uint32_t)(CH * kAChunk);
    // A: 16-byte chunk (c, kg) of voxel v at aS + c kAChunk + kg 2048 + v 16.
    const __nv_bfloat16 *xs = x + ((long long)(z + 1) * plane + P0) * CIN;
    for (int e = tid; e < CH * 2 * kConvM; e += 128) {
        const int c = e / (2 * kConvM), r = e % (2 * kConvM), kg = r & 1, v = r >> 1;
        cp_async16(aS + c * kAChunk + kg * (kConvM * 16) + v * 16, xs + (long long)v * CIN + c * 16 + kg * 8);
    }
    // B: 16-byte chunk (c, kg) of row n at bS + c kBChunk + kg N 16 + n 16.
    for (int e = tid; e < CH * 2 * N; e += 128) {
        const int c = e / (2 * N), r = e % (2 * N), kg = r & 1, n = r >> 1;
        cp_async16(bS + c * kBChunk + kg * (N * 16) + n * 16, w + (size_t)n * CIN + c * 16 + kg * 8);
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for (int c = 0; c < CH; ++c) {
#pragma unroll
            for (int h = 0; h < N / NMMA; ++h) {
                const uint64_t ad = umma_desc(aS + c * kAChunk, kConvM * 16, 128);
                const uint64_t bd = umma_desc(bS + c * kBChunk + h * NMMA * 16, N * 16, 128);
                const uint32_t accum = c > 0 ? 1u : 0u;
                asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                             " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                             ::"r"(tmem + (uint32_t)(h * NMMA)), "l"(ad), "l"(bd), "r"(idesc), "r"(accum)
                             : "memory");
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     ::"r"(smem_u32(&mbar)) : "memory");
    }
    // CTA-uniform outcome, so the .sync.aligned TMEM loads never run in a
    // divergent warp.
    const bool ok = __syncthreads_and(mbar_wait(smem_u32(&mbar), 0u, err)) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
        // warp w owns TMEM lanes 32w..32w+31 = voxels of the tile
        const long long Pv = P0 + 32 * warp + lane;
        const int yv = (int)(Pv / Wp), xv = (int)(Pv - (long long)yv * Wp);
        const bool inside = xv >= 1 && xv <= W && yv >= 1 && yv <= H;
        const int cx = xv - 1, cy = yv - 1;
        const long long Wf = 2LL * W + 2, Hf = 2LL * H + 2;
#pragma unroll 1
        for (int par = 0; par < 8; ++par) {
            const long long f = ((long long)(2 * z + (par >> 2) + 1) * Hf + (2 * cy + ((par >> 1) & 1) + 1)) * Wf +
                                (2 * cx + (par & 1) + 1);
#pragma unroll
            for (int n0 = 0; n0 < COUT; n0 += 16) {
                uint32_t r[16];
                const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(par * COUT + n0);
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                               "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
                               "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                             : "r"(taddr) : "memory");
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (inside) {
                    __nv_bfloat162 hv[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        hv[q] = __floats2bfloat162_rn(__uint_as_float(r[2 * q]) + __ldg(bias + n0 + 2 * q),
                                                      __uint_as_float(r[2 * q + 1]) + __ldg(bias + n0 + 2 * q + 1));
                    uint4 *dst = reinterpret_cast<uint4 *>(y + f * ys + n0);
                    dst[0] = *reinterpret_cast<uint4 *>(&hv[0]);
                    dst[1] = *reinterpret_cast<uint4 *>(&hv[4]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

template <int CIN, int COUT>
static cudaError_t launch_up_tc(int W, int H, int D, const __nv_bfloat16 *x, const __nv_bfloat16 *w,
                                const float *bias, __nv_bfloat16 *y, int ys, int *err, cudaStream_t st) {
    constexpr int smem = (CIN / 16) * 2 * kConvM * 16 + (CIN / 16) * 2 * (8 * COUT) * 16;
    cudaError_t e = cudaFuncSetAttribute(k_upconv_tc<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const long long interior = (long long)(W + 2) * H;
    const dim3 grid((unsigned)((interior + kConvM - 1) / kConvM), (unsigned)D);
    k_upconv_tc<CIN, COUT><<<grid, 128, smem, st>>>(W, H, D, x, w, bias, y, ys, err);
    return cudaGetLastError();
}

cudaError_t launch_upconv_tc(int W, int H, int D, int cin, int cout, const __nv_bfloat16 *x,
                             const __nv_bfloat16 *w, const float *bias, __nv_bfloat16 *y, int ys, int *err,
                             cudaStream_t st) {
    if (ys % 8 != 0) return cudaErrorInvalidValue;
    if (cin == 32 && cout == 16) return launch_up_tc<32, 16>(W, H, D, x, w, bias, y, ys, err, st);
    if (cin == 64 && cout == 32) return launch_up_tc<64, 32>(W, H, D, x, w, bias, y, ys, err, st);
    if (cin == 128 && cout == 64) return launch_up_tc<128, 64>(W, H, D, x, w, bias, y, ys, err, st);
    return cudaErrorNotSupported;
}

// ---------------------------------------------------------------------------
// Data gradient of the transposed convolution on the tensor cores:
//   gx[v][ci] = (x[v][ci] > 0) * sum over (par, co) of gy[fine(v, par)][co] * W[par][co][ci],
// a GEMM of M = 128 padded coarse voxels (the tile of k_upconv_tc), K =
// 8 COUT (parity, channel) and N = CIN.  A is gy gathered at the fine voxels
// in the K-major layout of the 3x3x3 kernels ([k group][voxel][8], zero for
// halo voxels); B is the BF16 weights in the MN-major layout ([ci group]
// [k][8], k rows 16 B apart), re-laid from [8][COUT][CIN] while staging.
// The parities go in chunks of PC (all 8, or 4 for 128 -> 64, so that a
// chunk fits in shared memory), each chunk's MMAs committed to the mbarrier
// and waited on (bounded) before the next chunk is staged.  The epilogue
// masks by the forward activation and stores BF16.
// ---------------------------------------------------------------------------
template <int CIN, int COUT>
struct UpDgradShape {
    static constexpr int PC = CIN == 128 ? 4 : 8;         // parities per chunk
    static constexpr int KC = PC * COUT;                   // K per chunk
    static constexpr int ABYTES = KC * kConvM * 2;         // KC / 8 slabs of 128 voxels x 16 B
    static constexpr int BBYTES = KC * CIN * 2;
    static constexpr int SMEM = ABYTES + BBYTES;
    static_assert(SMEM <= 227 * 1024, "chunk exceeds shared memory");
    static_assert(CIN % 16 == 0 && CIN <= 256, "N = CIN must be a multiple of 16, at most 256");
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(128, 1)
k_upconv_dgrad_tc(int W, int H, int D, const __nv_bfloat16 *__restrict__ gy, int gs,
                  const __nv_bfloat16 *__restrict__ w, const __nv_bfloat16 *__restrict__ act,
                  __nv_bfloat16 *__restrict__ gx, int *err) {
    using S = UpDgradShape<CIN, COUT>;
    constexpr int KC = S::KC, NG = COUT / 8;
    // kind::f16, D FP32, A and B BF16, A K-major, B MN-major
    constexpr uint32_t idesc = umma_idesc_bf16(kConvM, CIN) | (1u << 16);
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int Wp = W + 2, Hp = H + 2;
    const long long plane = (long long)Wp * Hp;
    const int z = blockIdx.y;                                              // interior coarse plane
    const long long P0 = (long long)Wp + (long long)kConvM * blockIdx.x;   // first voxel of the tile

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base)), "r"(CIN < 32 ? 32 : CIN) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    const uint32_t aS = smem_u32(smem), bS = aS + (uint32_t)S::ABYTES;
    // thread tid gathers voxel P0 + tid of the tile
    const long long P = P0 + tid;
    const int yv = (int)(P / Wp), xv = (int)(P - (long long)yv * Wp);
    const bool inside = xv >= 1 && xv <= W && yv >= 1 && yv <= H;
    const long long Wf = 2LL * W + 2, Hf = 2LL * H + 2;
    bool ok = true;
    constexpr int NCH = 8 / S::PC;
#pragma unroll 1
    for (int c = 0; c < NCH && ok; ++c) {
        // A: k group kg = (parity, 8 channels) of voxel tid at aS + kg 2048 + tid 16
#pragma unroll 4
        for (int kg = 0; kg < KC / 8; ++kg) {
            const int par = c * S::PC + kg / NG, g = kg % NG;
            const uint32_t dst = aS + kg * (kConvM * 16) + tid * 16;
            if (inside) {
                const long long f = ((long long)(2 * z + (par >> 2) + 1) * Hf + (2 * (yv - 1) + ((par >> 1) & 1) + 1)) * Wf +
                                    (2 * (xv - 1) + (par & 1) + 1);
                cp_async16(dst, gy + f * gs + g * 8);
            } else {
                st_shared_zero16(dst);
            }
        }
        // B: chunk (k, ci group ng) of W row c KC + k at bS + (ng KC + k) 16
        for (int e = tid; e < KC * (CIN / 8); e += 128) {
            const int k = e / (CIN / 8), ng = e % (CIN / 8);
            cp_async16(bS + (ng * KC + k) * 16, w + (size_t)(c * KC + k) * CIN + ng * 8);
        }
        asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint64_t ad0 = umma_desc(aS, kConvM * 16, 128), bd0 = umma_desc(bS, 128, KC * 16);
#pragma unroll
            for (int s = 0; s < KC / 16; ++s) {
                const uint64_t ad = ad0 + (uint64_t)((2 * s * kConvM * 16) >> 4);
                const uint64_t bd = bd0 + (uint64_t)((s * 256) >> 4);
                const uint32_t accum = (c > 0 || s > 0) ? 1u : 0u;
                asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                             " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                             ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(accum) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(&mbar)) : "memory");
        }
        // The staged chunk is overwritten only once its MMAs completed.
        ok = __syncthreads_and(mbar_wait(smem_u32(&mbar), (uint32_t)(c & 1), err)) != 0;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
        // TMEM lane tid = 32 warp + lane is this thread's own voxel P
        const long long vc = (long long)(z + 1) * plane + P;
#pragma unroll 1
        for (int n0 = 0; n0 < CIN; n0 += 16) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)n0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
                           "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                         : "r"(taddr) : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (inside) {
                const uint4 a0 = __ldg(reinterpret_cast<const uint4 *>(act + vc * CIN + n0));
                const uint4 a1 = __ldg(reinterpret_cast<const uint4 *>(act + vc * CIN + n0) + 1);
                const __nv_bfloat16 *ah0 = reinterpret_cast<const __nv_bfloat16 *>(&a0);
                const __nv_bfloat16 *ah1 = reinterpret_cast<const __nv_bfloat16 *>(&a1);
                __nv_bfloat162 hv[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const float a = __bfloat162float(q < 4 ? ah0[2 * q] : ah1[2 * q - 8]) > 0.0f
                                        ? __uint_as_float(r[2 * q]) : 0.0f;
                    const float b = __bfloat162float(q < 4 ? ah0[2 * q + 1] : ah1[2 * q - 7]) > 0.0f
                                        ? __uint_as_float(r[2 * q + 1]) : 0.0f;
                    hv[q] = __floats2bfloat162_rn(a, b);
                }
                uint4 *dst = reinterpret_cast<uint4 *>(gx + vc * CIN + n0);
                dst[0] = *reinterpret_cast<uint4 *>(&hv[0]);
                dst[1] = *reinterpret_cast<uint4 *>(&hv[4]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(CIN < 32 ? 32 : CIN)
                     : "memory");
}

template <int CIN, int COUT>
static cudaError_t launch_up_dgrad(int W, int H, int D, const __nv_bfloat16 *gy, int gs, const __nv_bfloat16 *w,
                                   const __nv_bfloat16 *act, __nv_bfloat16 *gx, int *err, cudaStream_t st) {
    constexpr int smem = UpDgradShape<CIN, COUT>::SMEM;
    cudaError_t e = cudaFuncSetAttribute(k_upconv_dgrad_tc<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem);
    if (e != cudaSuccess) return e;
    const long long interior = (long long)(W + 2) * H;
    const dim3 grid((unsigned)((interior + kConvM - 1) / kConvM), (unsigned)D);
    k_upconv_dgrad_tc<CIN, COUT><<<grid, 128, smem, st>>>(W, H, D, gy, gs, w, act, gx, err);
    return cudaGetLastError();
}

cudaError_t launch_upconv_dgrad_tc(int W, int H, int D, int cin, int cout, const __nv_bfloat16 *gy, int gs,
                                   const __nv_bfloat16 *w, const __nv_bfloat16 *act, __nv_bfloat16 *gx, int *err,
                                   cudaStream_t st) {
    if (gs % 8 != 0) return cudaErrorInvalidValue;
    if (cin == 32 && cout == 16) return launch_up_dgrad<32, 16>(W, H, D, gy, gs, w, act, gx, err, st);
    if (cin == 64 && cout == 32) return launch_up_dgrad<64, 32>(W, H, D, gy, gs, w, act, gx, err, st);
    if (cin == 128 && cout == 64) return launch_up_dgrad<128, 64>(W, H, D, gy, gs, w, act, gx, err, st);
    return cudaErrorNotSupported;
}

// ---------------------------------------------------------------------------
// Weight gradients on the tensor cores.  For the 3x3x3 convolution
//   dW[tap][co][ci] = sum over voxels P of gy[P][co] * x[P + off(tap)][ci],
// a GEMM whose reduction (K) runs over voxels.  Both tensors are channels
// last, so 8 channels of one voxel are one 16-byte row, and a block of
// voxels staged row by row is already an operand in the MN-major, no-swizzle
// layout: core matrices of 8 voxels (K) x 8 channels (M or N), 8-voxel groups
// LBO = 128 B apart, 8-channel groups SBO apart.  With K blocks of KB voxels:
//   A (M = 128): 16 eight-channel groups (r, g) of x over the 9 row offsets
//     r = (dz, dy), each a window of KB + 2 voxels staged from one voxel
//     early; tap dx reads the same window 16 * (dx + 1) bytes further on;
//   B (N = Cout): gy over the KB voxels;
//   three accumulators (dx) of Cout columns in TMEM.
// The K range is the padded voxels from the first interior row to the last;
// gy is zero on the halo, so halo voxels add nothing.  For the 2x2x2
// transposed convolution (8 parities)
//   dW[par][co][ci] = sum over coarse voxels v of gy[fine(v, par)][co] * x[v][ci]:
//   A (M = 128): 16 groups (par, co group) of gy gathered at the fine voxels
//     (zero for halo voxels), B (N = Cin): x over the KB coarse voxels.
// A CTA owns one M tile (blockIdx.y) and a run of K blocks (blockIdx.x),
// double buffered: block i + 1 is staged by cp.async before the MMAs of block
// i are issued, so its loads are in flight while they run (issuing the MMAs
// first exposes every block's load latency and measured 10 % slower).  One
// thread issues the MMAs; each buffer's commit arrives on its own mbarrier,
// waited on (bounded in time) before the buffer is restaged.  The CTA's sums
// are added to dW with FP32 atomics.
// ---------------------------------------------------------------------------
constexpr int kWgKB = 128;                 // voxels per K block; the up gather has one per thread
static_assert(kWgKB + 2 <= BLZ_CONV_SLACK, "the last K block's window must stay inside the slack");

struct WgTcArgs {
    const __nv_bfloat16 *x;
    int xs;                                // layer input (conv) / coarse input (up), channel stride
    const __nv_bfloat16 *gy;
    int gys, gyoff;                        // output gradient: channel stride, first channel
    int W, H, D;                           // dims of the K loop's level (up: the coarse one)
    long long pbeg;                        // first padded voxel of the K range
    int nkb, kb_per;                       // K blocks in all, per CTA
    float *dw;
    int *err;
};

template <int MODE, int CIN, int CO>
struct WgShape {
    static constexpr int AW = MODE == 0 ? kWgKB + 2 : kWgKB;   // staged voxels per A group
    static constexpr int GA = AW * 16;                         // bytes per A group
    static constexpr int NGA = (MODE == 0 ? CIN : CO) / 8;     // A groups per row offset / parity
    static constexpr int NGALL = (MODE == 0 ? 9 : 8) * NGA;
    static constexpr int MTILES = (NGALL + 15) / 16;
    static constexpr int N = MODE == 0 ? CO : CIN;
    static constexpr int NGB = N / 8;
    static constexpr int GB = kWgKB * 16;
    static constexpr int ABYTES = 16 * GA, BUF = ABYTES + NGB * GB;
    static constexpr int NACC = MODE == 0 ? 3 : 1;
    static constexpr int COLS = NACC * N <= 32 ? 32 : NACC * N <= 64 ? 64 : NACC * N <= 128 ? 128
                                                    : NACC * N <= 256 ? 256 : 512;
    static_assert(NACC * N <= 512, "accumulators exceed tensor memory");
    static_assert(N % 16 == 0 && N <= 256, "MN-major B needs N a multiple of 16, at most 256");
};

template <int MODE, int CIN, int CO>
__global__ void __launch_bounds__(128, 1) k_wgrad_tc(WgTcArgs a) {
    using S = WgShape<MODE, CIN, CO>;
    constexpr int KB = kWgKB, N = S::N, NGA = S::NGA;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mt = blockIdx.y;
    const long long Wp = a.W + 2, Hp = a.H + 2, plane = Wp * Hp;
    const int kb0 = blockIdx.x * a.kb_per;
    const int nk = min(a.kb_per, a.nkb - kb0);
    const uint32_t s0 = smem_u32(smem);
    const uint32_t mb0 = smem_u32(&mbar[0]);
    auto mb = [&](int b) { return mb0 + 8u * (uint32_t)b; };

    // A groups that hold no row (conv tiles past the 9th row offset) stay zero.
    for (int e = tid; e < 2 * S::BUF / 16; e += 128) st_shared_zero16(s0 + e * 16);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base)), "r"(S::COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb(0)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb(1)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    auto stage = [&](int kb, int buf) {
        const uint32_t sa = s0 + buf * S::BUF, sb = sa + S::ABYTES;
        const long long P0 = a.pbeg + (long long)kb * KB;
        if constexpr (MODE == 0) {
            // local row offset lr holds groups lr * NGA .. lr * NGA + NGA - 1;
            // element e of its window is voxel e / NGA, group e % NGA
            constexpr int NR = 16 / NGA, PER = S::AW * NGA;
#pragma unroll
            for (int lr = 0; lr < NR; ++lr) {
                const int r = mt * NR + lr;
                if (r >= 9) break;
                const __nv_bfloat16 *src =
                    a.x + (P0 - 1 + (long long)(r / 3 - 1) * plane + (long long)(r % 3 - 1) * Wp) * a.xs;
                for (int e = tid; e < PER; e += 128) {
                    const int v = e / NGA, g = e & (NGA - 1);
                    cp_async16(sa + (lr * NGA + g) * S::GA + v * 16, src + v * a.xs + g * 8);
                }
            }
            const __nv_bfloat16 *gb = a.gy + P0 * a.gys + a.gyoff;
            for (int e = tid; e < S::NGB * KB; e += 128) {
                const int g = e & (S::NGB - 1), v = e / S::NGB;
                cp_async16(sb + g * S::GB + v * 16, gb + v * a.gys + g * 8);
            }
        } else {
            // thread tid gathers coarse voxel P0 + tid's 16 groups
            const long long P = P0 + tid;
            const long long zc = P / plane, rem = P - zc * plane;
            const long long yc = rem / Wp, xc = rem - yc * Wp;
            const bool inside = zc >= 1 && zc <= a.D && yc >= 1 && yc <= a.H && xc >= 1 && xc <= a.W;
            const long long Wf = 2LL * a.W + 2, Hf = 2LL * a.H + 2;
#pragma unroll 4
            for (int lg = 0; lg < 16; ++lg) {
                const int grp = mt * 16 + lg, par = grp / NGA, g = grp % NGA;
                const uint32_t dst = sa + lg * S::GA + tid * 16;
                if (inside) {
                    const long long f = ((2 * zc - 1 + (par >> 2)) * Hf + (2 * yc - 1 + ((par >> 1) & 1))) * Wf +
                                        (2 * xc - 1 + (par & 1));
                    cp_async16(dst, a.gy + f * a.gys + a.gyoff + g * 8);
                } else {
                    st_shared_zero16(dst);
                }
            }
            for (int e = tid; e < S::NGB * KB; e += 128) {
                const int g = e % S::NGB, v = e / S::NGB;
                cp_async16(sb + g * S::GB + v * 16, a.x + (P0 + v) * a.xs + g * 8);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };

    // kind::f16, D FP32, A and B BF16, both MN-major
    constexpr uint32_t idesc = umma_idesc_bf16(128, N) | (1u << 15) | (1u << 16);
    bool ok = true;
    int issued = 0;                                      // MMA batches committed
    if (nk > 0) stage(kb0, 0);
    for (int i = 0; i < nk; ++i) {
        const int buf = i & 1;
        if (i + 1 < nk) {
            // buffer buf ^ 1 was last read by the MMAs of block i - 1
            if (i >= 1) ok = __syncthreads_and(mbar_wait(mb(buf ^ 1), ((i - 1) >> 1) & 1, a.err)) != 0;
            if (!ok) break;
            stage(kb0 + i + 1, buf ^ 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = s0 + buf * S::BUF, sb = sa + S::ABYTES;
            const uint64_t ad0 = umma_desc(sa, 128, S::GA), bd0 = umma_desc(sb, 128, S::GB);
#pragma unroll
            for (int kk = 0; kk < KB / 16; ++kk) {
                const uint64_t bd = bd0 + (uint64_t)((kk * 256) >> 4);
#pragma unroll
                for (int d = 0; d < S::NACC; ++d) {
                    const uint64_t ad = ad0 + (uint64_t)((kk * 256 + (MODE == 0 ? d * 16 : 0)) >> 4);
                    const uint32_t acc = (i > 0 || kk > 0) ? 1u : 0u;
                    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                                 " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                                 ::"r"(tmem + (uint32_t)(d * N)), "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                                 : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(mb(buf)) : "memory");
        }
        ++issued;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    // The last commit completes after every MMA issued before it.
    if (issued > 0)
        ok = __syncthreads_and(mbar_wait(mb((issued - 1) & 1), ((issued - 1) >> 1) & 1, a.err) && ok) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok && issued == nk && nk > 0) {
        // TMEM lane m = A row: group m / 8, channel m % 8 of it.
        const int m = 32 * warp + lane, grp = mt * 16 + (m >> 3), c8 = m & 7;
        const bool valid = grp < S::NGALL;
        const int hi = grp / NGA, ch = (grp % NGA) * 8 + c8;   // conv: (row offset, ci); up: (parity, co)
#pragma unroll 1
        for (int d = 0; d < S::NACC; ++d) {
#pragma unroll 1
            for (int n0 = 0; n0 < N; n0 += 16) {
                uint32_t r[16];
                const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(d * N + n0);
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                               "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
                               "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                             : "r"(taddr) : "memory");
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (valid) {
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        const int n = n0 + q;
                        const size_t o = MODE == 0 ? ((size_t)(3 * hi + d) * CO + n) * CIN + ch
                                                   : ((size_t)hi * CO + ch) * CIN + n;
                        atomicAdd(a.dw + o, __uint_as_float(r[q]));
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::COLS) : "memory");
}

template <int MODE, int CIN, int CO>
static cudaError_t launch_wg_tc(WgTcArgs a, cudaStream_t st) {
    using S = WgShape<MODE, CIN, CO>;
    constexpr int smem = 2 * S::BUF;
    cudaError_t e = cudaFuncSetAttribute(k_wgrad_tc<MODE, CIN, CO>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const long long Wp = a.W + 2, plane = Wp * (a.H + 2);
    a.pbeg = plane + Wp;                                  // first interior row
    const long long pend = (long long)(a.D + 1) * plane - Wp;   // past the last interior row
    const long long nkb = (pend - a.pbeg + kWgKB - 1) / kWgKB;
    if (nkb >= (1LL << 30)) return cudaErrorInvalidValue;
    // about two CTAs per SM, at least four K blocks each
    const long long want = (2 * 148 + S::MTILES - 1) / S::MTILES;
    long long per = (nkb + want - 1) / want;
    if (per < 4) per = 4;
    a.nkb = (int)nkb;
    a.kb_per = (int)per;
    const dim3 grid((unsigned)((nkb + per - 1) / per), (unsigned)S::MTILES);
    k_wgrad_tc<MODE, CIN, CO><<<grid, 128, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_wgrad_tc(int up, int W, int H, int D, int cin, int cout, const __nv_bfloat16 *x, int xs,
                            const __nv_bfloat16 *gy, int gys, int gyoff, float *dw, int *err, cudaStream_t st) {
    if (xs % 8 != 0 || gys % 8 != 0 || gyoff % 8 != 0) return cudaErrorInvalidValue;
    WgTcArgs a{x, xs, gy, gys, gyoff, W, H, D, 0, 0, 0, dw, err};
    if (up) {
        if (cin == 32 && cout == 16) return launch_wg_tc<1, 32, 16>(a, st);
        if (cin == 64 && cout == 32) return launch_wg_tc<1, 64, 32>(a, st);
        if (cin == 128 && cout == 64) return launch_wg_tc<1, 128, 64>(a, st);
        return cudaErrorNotSupported;
    }
#define BLZ_WG(ci, co) if (cin == ci && cout == co) return launch_wg_tc<0, ci, co>(a, st)
    BLZ_WG(16, 16); BLZ_WG(16, 32); BLZ_WG(32, 16); BLZ_WG(32, 32); BLZ_WG(32, 64);
    BLZ_WG(64, 32); BLZ_WG(64, 64); BLZ_WG(64, 128); BLZ_WG(128, 64); BLZ_WG(128, 128);
#undef BLZ_WG
    return cudaErrorNotSupported;
}

} // namespace blz

namespace {
__device__ int g_conv_timeout;          // set by a convolution whose MMA wait gave up
}

extern "C" int blz_conv3d(const blz_conv_desc *d, const void *x, const void *w, const float *bias, void *y,
                          void *cuda_stream) {
    using namespace blz;
    if (!d || !x || !w || !bias || !y) return BLZ_ERR_ARG;
    if (d->W < 1 || d->H < 1 || d->D < 1 || d->cin <= 0 || d->cin % 16 ||
        (d->cout != 16 && d->cout != 32 && d->cout != 64 && d->cout != 128)) {
        set_thread_error("blz_conv3d: need cin % 16 == 0 and cout in {16, 32, 64, 128}");
        return BLZ_ERR_ARG;
    }
    int *flag = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&flag, g_conv_timeout);
    if (e == cudaSuccess) e = cudaMemsetAsync(flag, 0, sizeof(int), (cudaStream_t)cuda_stream);
    const ConvDesc cd{d->W, d->H, d->D, d->cin, d->cout, d->relu, d->out_f32, d->cout, 0};
    if (e == cudaSuccess)
        e = launch_conv3d(cd, static_cast<const __nv_bfloat16 *>(x), static_cast<const __nv_bfloat16 *>(w), bias, y,
                          flag, (cudaStream_t)cuda_stream);
    int timeout = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&timeout, flag, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)cuda_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)cuda_stream);
    if (e != cudaSuccess) {
        set_thread_error(cudaGetErrorString(e));
        return BLZ_ERR_CUDA;
    }
    if (timeout) {
        set_thread_error("blz_conv3d: tensor-core completion wait timed out");
        return BLZ_ERR_TIMEOUT;
    }
    return BLZ_OK;
}
