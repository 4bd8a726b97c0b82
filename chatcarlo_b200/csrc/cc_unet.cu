// BF16 tensor-core kernels of the 3D U-Net kerma denoiser (sm_100a).
//
// Activations are channels-last BF16 tensors [B, D, H, W, C] with C a
// multiple of 16.  Every 3x3x3 "same" convolution is an implicit GEMM on the
// 5th-generation tensor cores:
//
//   D[v, co] = sum_{tap, ci} X[v + off(tap), ci] * W[tap, co, ci]
//
// M = 128 output voxels per CTA, N = output channels, K = 27 taps x input
// channels.  All 256 threads of the CTA gather the A tile (neighbour voxel
// rows, zero outside the volume) and the B tile (weights of one tap) into
// shared memory in the K-major, no-swizzle canonical layout; one thread
// issues tcgen05.mma (kind::f16, BF16 inputs, FP32 accumulator in tensor
// memory) and commits to an mbarrier, so the gather of the next stage runs
// while the tensor core works on the current one (two stages).  The
// epilogue reads the accumulator back with tcgen05.ld and applies bias and
// ReLU (forward) or the ReLU mask of the layer below (backward data).
//
// A convolution input may be the channel concatenation of a full-resolution
// tensor a and a half-resolution tensor b read nearest-upsampled (the U-Net
// decoder's skip + upsampled path), fused into the gather.
//
// The weight gradient is a second GEMM with M = 27 x C_in rows (tap, ci),
// N = C_out and K = voxels, its operands MN-major in shared memory, split
// over voxel ranges and reduced with FP32 atomics.
//
// Every mbarrier wait is bounded by the global timer; a wait that runs out
// sets a status bit that the host reads, and the CTA still frees its tensor
// memory before it returns.
#include <algorithm>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>

#include <mutex>
#include <string>

#include "../../include/chatcarlo_b200_unet.h"

namespace {

constexpr int TILE_M = 128;
constexpr int THREADS = 256;
constexpr int KSTAGE = 64;                  // voxels per weight-gradient pipeline stage
constexpr unsigned long long WAIT_NS = 2000000000ull;   // 2 s bound on every mbarrier wait

__device__ unsigned g_status;               // bit 0: an mbarrier wait ran out

thread_local std::string t_err;

int set_error(int code, const std::string& msg) {
    t_err = msg;
    return code;
}

#define CU_CHECK(call)                                                               \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) return set_error(CCU_E_DEVICE, cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the completion of the phase with this parity, at most WAIT_NS.
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > WAIT_NS) return false;
    }
}

// One arrival on an mbarrier (release semantics, CTA scope).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
                 : "memory");
}

// mbar_wait that also gives up once another thread of the CTA has set
// *fail (its own wait ran out); sets *fail itself when its WAIT_NS run out.
__device__ bool mbar_wait_or_fail(uint64_t* bar, uint32_t parity, volatile int* fail) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*fail) return false;
        if (global_ns() - t0 > WAIT_NS) {
            *fail = 1;
            return false;
        }
    }
}

// The mbarrier receives one arrival when all of this thread's earlier
// cp.async copies have landed (the arrival is not counted in advance: the
// barrier's expected count includes it).
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// One arrival on an mbarrier that also raises the bytes its phase waits
// for by `bytes` (the tensor-memory-accelerator copies that complete on it).
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Tile load of one box of a 5D tensor map into this CTA's shared memory,
// completing on an mbarrier (no multicast).  Coordinates outside the tensor
// read zeros; the innermost coordinate must be 16-byte aligned.
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2, int c3, int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
        "%6}], [%7];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Tensor memory: a power of two >= 32 columns, allocated by one whole warp.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Shared-memory matrix descriptor, no swizzle: start, leading-dimension
// byte offset (between core matrices adjacent in K), stride-dimension byte
// offset (between core matrices adjacent in M/N), descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// The same with a swizzled layout: type 6 (32-byte rows), 4 (64) or 2 (128),
// bits 61-63; for MN-major operands lbo is then the byte offset between
// swizzle-atom columns along M/N and sbo between groups of 8 rows along K.
__device__ __forceinline__ uint64_t smem_desc_sw(uint32_t addr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
    return smem_desc(addr, lbo, sbo) | ((uint64_t)(layout & 7u) << 61);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B,
// A/B K-major (0) or MN-major (1), N >> 3, M >> 4.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 lanes x 8 consecutive 32-bit columns; lane quarter in bits 31:16.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float f[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 8; ++j) f[j] = __uint_as_float(r[j]);
}

// tmem_ld8 without the wait: several loads in flight, then tmem_wait_ld()
__device__ __forceinline__ void tmem_ld8_nw(uint32_t taddr, uint32_t r[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint4 pack_bf16x8(const float f[8]) {
    uint4 u;
    __nv_bfloat162 h0 = __floats2bfloat162_rn(f[0], f[1]), h1 = __floats2bfloat162_rn(f[2], f[3]);
    __nv_bfloat162 h2 = __floats2bfloat162_rn(f[4], f[5]), h3 = __floats2bfloat162_rn(f[6], f[7]);
    memcpy(&u.x, &h0, 4);
    memcpy(&u.y, &h1, 4);
    memcpy(&u.z, &h2, 4);
    memcpy(&u.w, &h3, 4);
    return u;
}

__device__ __forceinline__ void unpack_bf16x8(uint4 u, float f[8]) {
    __nv_bfloat162 h[4];
    memcpy(&h[0], &u.x, 4);
    memcpy(&h[1], &u.y, 4);
    memcpy(&h[2], &u.z, 4);
    memcpy(&h[3], &u.w, 4);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float2 t = __bfloat1622float2(h[j]);
        f[2 * j] = t.x;
        f[2 * j + 1] = t.y;
    }
}

// ---------------------------------------------------------------------------
// convolution input: a (full resolution) ++ b (half resolution, upsampled)
// ---------------------------------------------------------------------------

struct Src {
    const __nv_bfloat16* a;
    const __nv_bfloat16* b;
    int ca, cb;
    int B, D, H, W;
};

__device__ __forceinline__ void voxel_coords(long long v, const Src& s, int& n, int& z, int& y, int& x) {
    x = (int)(v % s.W);
    long long t = v / s.W;
    y = (int)(t % s.H);
    t /= s.H;
    z = (int)(t % s.D);
    n = (int)(t / s.D);
}

// ---------------------------------------------------------------------------
// gather machinery shared by the two GEMM kernels
// ---------------------------------------------------------------------------

// 16-byte asynchronous copy global -> shared; src_bytes 0 writes zeros
// (the zero padding outside the volume) without reading src.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
// cp_async16 that bypasses L1 (cached in L2 only): for streamed data read
// once per CTA, where shared memory leaves L1 little room
__device__ __forceinline__ void cp_async16_cg(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory");
}

// A voxel of a tile: flattened index (-1 outside the range), boundary
// flags (bit 0 z > 0, 1 z < D-1, 2 y > 0, 3 y < H-1, 4 x > 0, 5 x < W-1),
// and for the half-resolution source its coarse voxel index and the
// parities of its coordinates (bit 0 x, 1 y, 2 z).
struct VoxRec {
    int v, flags, cv, par;
};

__device__ __forceinline__ VoxRec make_vox(long long v, long long n_vox, const Src& s) {
    VoxRec r{-1, 0, 0, 0};
    if (v < n_vox) {
        int n, z, y, x;
        voxel_coords(v, s, n, z, y, x);
        r.v = (int)v;
        r.flags = (z > 0) | ((z < s.D - 1) << 1) | ((y > 0) << 2) | ((y < s.H - 1) << 3) | ((x > 0) << 4) |
                  ((x < s.W - 1) << 5);
        if (s.cb) {
            r.cv = ((n * (s.D >> 1) + (z >> 1)) * (s.H >> 1) + (y >> 1)) * (s.W >> 1) + (x >> 1);
            r.par = (x & 1) | ((y & 1) << 1) | ((z & 1) << 2);
        }
    }
    return r;
}

// Boundary flags a voxel needs for its neighbour at tap to lie inside.
__host__ __device__ constexpr int tap_req(int t) {
    return (t / 9 == 0 ? 1 : 0) | (t / 9 == 2 ? 2 : 0) | ((t / 3) % 3 == 0 ? 4 : 0) | ((t / 3) % 3 == 2 ? 8 : 0) |
           (t % 3 == 0 ? 16 : 0) | (t % 3 == 2 ? 32 : 0);
}

// Offset (in coarse voxels) of the coarse voxel holding the neighbour at
// tap of a fine voxel with coordinate parities par: the coarse coordinate
// moves by floor((parity + d) / 2) along each axis.
__device__ __forceinline__ int coarse_offset(const Src& s, int par, int tap) {
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    const int cz = (((par >> 2) & 1) + dz) >> 1, cy = (((par >> 1) & 1) + dy) >> 1, cx = ((par & 1) + dx) >> 1;
    return (cz * (s.H >> 1) + cy) * (s.W >> 1) + cx;
}

// ---------------------------------------------------------------------------
// forward / backward-data convolution
// ---------------------------------------------------------------------------

constexpr int KS = 64;                      // K elements (tap x channel) per convolution stage

struct ConvP {
    Src src;
    const __nv_bfloat16* w;      // packed in tile order: packed_elems(N, cin)
    const float* bias;           // [N] or null
    int relu;
    long long n_vox;
    // output channels [0, split) -> out0 [v][split], masked by mask0 (same
    // layout) when given; channels [split, N) -> out1 [v][N - split]
    __nv_bfloat16* out0;
    const __nv_bfloat16* mask0;
    int split;
    __nv_bfloat16* out1;
    // the network's 1 x 1 x 1 head on a 16-channel layer (plane-stationary
    // kernel only): head_out[v] = head_x[v] + head[16] + sum_j head[j] a_j,
    // a_j the BF16 activations; out0 may then be null (not stored)
    const float* head;
    const float* head_x;
    float* head_out;
};

// Bias, ReLU, mask and BF16 store of output channels [c0, c0 + 8) of voxel v
// (f returns the activations before the BF16 rounding).
__device__ __forceinline__ void conv_store(const ConvP& P, long long v, int c0, int n_out, float f[8]) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (P.bias) f[j] += __ldg(P.bias + c0 + j);
        if (P.relu) f[j] = fmaxf(f[j], 0.0f);
    }
    if (c0 < P.split) {
        const size_t o = (size_t)v * P.split + c0;
        if (P.mask0) {
            float mk[8];
            unpack_bf16x8(__ldg(reinterpret_cast<const uint4*>(P.mask0 + o)), mk);
#pragma unroll
            for (int j = 0; j < 8; ++j) f[j] = mk[j] > 0.0f ? f[j] : 0.0f;
        }
        if (P.out0) *reinterpret_cast<uint4*>(P.out0 + o) = pack_bf16x8(f);
    } else {
        const size_t o = (size_t)v * (n_out - P.split) + (c0 - P.split);
        *reinterpret_cast<uint4*>(P.out1 + o) = pack_bf16x8(f);
    }
}

__host__ __device__ constexpr uint32_t tmem_cols(int n) {
    return n <= 32 ? 32u : (n <= 64 ? 64u : (n <= 128 ? 128u : 256u));
}

constexpr int CONV_STAGES = 3;
__host__ __device__ constexpr uint32_t conv_stage_bytes(int n) { return (uint32_t)(TILE_M + n) * KS * 2; }

// Weights packed in shared-memory tile order: stage s (K elements
// [64 s, 64 s + 64) of 27 x c, k = tap * c + ch), chunk c8 of 8 elements,
// output row r: element ((s * 8 + c8) * n + r) * 8 + e, zero beyond 27 x c.
__host__ __device__ constexpr long long packed_elems(int n, int c) {
    return (long long)((27 * c + KS - 1) / KS) * n * KS;
}

// K runs over (tap, channel) in stages of KS elements; a stage's A tile is
// the 128 output voxels' neighbours for those (tap, channel) pairs, its B
// tile the matching packed weights.  CONV_STAGES stages are in flight:
// cp.async fills stage s + 2 while the tensor core works on stage s.  Each
// thread gathers for one output row (m = tid % 128) four chunks per stage
// (c8 = tid / 128 + 2 j) and steps their (tap, channel) incrementally.
template <int N>
__global__ void __launch_bounds__(THREADS) conv_kernel(const ConvP P) {
    constexpr int NS = CONV_STAGES;
    constexpr uint32_t A_BYTES = TILE_M * KS * 2, STAGE = conv_stage_bytes(N);
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ uint64_t bar[NS];
    __shared__ uint32_t s_tmem;
    __shared__ int s_off[27];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Src& S = P.src;
    const int cin = S.ca + S.cb;
    const int n_stages = (27 * cin + KS - 1) / KS;
    const long long m0 = (long long)blockIdx.x * TILE_M;

    if (tid < 27) {
        const int dz = tid / 9 - 1, dy = (tid / 3) % 3 - 1, dx = tid % 3 - 1;
        s_off[tid] = ((dz * S.H + dy) * S.W + dx) * S.ca;          // element offset in a
    }
    if (warp == 0) tmem_alloc(&s_tmem, tmem_cols(N));
    if (tid == 0) {
        for (int i = 0; i < NS; ++i) mbar_init(&bar[i], 1);
        mbar_init_fence();
    }
    // this thread's output row
    const int m = tid & (TILE_M - 1), c8_0 = tid >> 7;
    const VoxRec row = make_vox(m0 + m, P.n_vox, S);
    uint32_t valid = 0;                              // taps whose neighbour lies inside the volume
    if (row.v >= 0) {
#pragma unroll
        for (int t = 0; t < 27; ++t)
            if ((row.flags & tap_req(t)) == tap_req(t)) valid |= 1u << t;
    }
    const __nv_bfloat16* a_row = S.a + (size_t)(row.v < 0 ? 0 : row.v) * S.ca;
    const __nv_bfloat16* b_row = S.cb ? S.b + (size_t)row.cv * S.cb : S.b;
    // (tap, ch) of this thread's 4 chunks in stage 0; a stage advances K by KS
    int tap[4], ch[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int k = (c8_0 + 2 * j) * 8;
        tap[j] = k / cin;
        ch[j] = k - tap[j] * cin;
    }
    const int step_tap = KS / cin, step_ch = KS - (KS / cin) * cin;
    uint32_t dstA[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) dstA[j] = (c8_0 + 2 * j) * (TILE_M * 16) + (m >> 3) * 128 + (m & 7) * 16;

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t sbase = smem_u32(smem);
    constexpr uint32_t IDESC = idesc_bf16(TILE_M, N, 0, 0);

    // copies of stage s; called for s = 0, 1, 2, ... in order
    auto issue = [&](int s) {
        const uint32_t sa = sbase + (uint32_t)(s % NS) * STAGE, sb = sa + A_BYTES;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int t = tap[j], c = ch[j];
            uint32_t bytes = 0;
            const void* src = S.a;
            if ((valid >> t) & 1u) {                 // t <= 27, and bit 27 is never set
                bytes = 16;
                src = c < S.ca ? (const void*)(a_row + s_off[t] + c)
                               : (const void*)(b_row + (size_t)coarse_offset(S, row.par, t) * S.cb + (c - S.ca));
            }
            cp_async16(sa + dstA[j], src, bytes);
            int nc = c + step_ch, nt = t + step_tap;
            if (nc >= cin) {
                nc -= cin;
                ++nt;
            }
            tap[j] = nt;
            ch[j] = nc;
        }
        const __nv_bfloat16* wb = P.w + (size_t)s * (N * KS);
        for (int i = tid; i < N * (KS / 8); i += THREADS) cp_async16(sb + i * 16, wb + (size_t)i * 8, 16u);
    };

    bool ok = true;
    int issued = 0;                                  // stages whose MMAs were committed
    for (int s = 0; s < NS - 1; ++s) {
        if (s < n_stages) issue(s);
        cp_async_commit();
    }
    for (int it = 0; it < n_stages; ++it) {
        cp_async_wait<NS - 2>();                     // this thread's copies of stage it landed
        fence_proxy_async();                         // ... and are visible to the tensor core
        if (!__syncthreads_and(ok)) { ok = false; break; }
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = sbase + (uint32_t)(it % NS) * STAGE, b0 = a0 + A_BYTES;
#pragma unroll
            for (int k = 0; k < KS / 16; ++k) {
                uint64_t ad = smem_desc(a0 + k * 2 * (TILE_M * 16), TILE_M * 16, 128);
                uint64_t bd = smem_desc(b0 + k * 2 * (N * 16), N * 16, 128);
                mma_bf16(tmem, ad, bd, IDESC, (it > 0 || k > 0) ? 1u : 0u);
            }
            mma_commit(&bar[it % NS]);
        }
        issued = it + 1;
        // stage it + NS - 1 reuses the buffer that the MMAs of stage it - 1 read
        const int nxt = it + NS - 1;
        if (nxt < n_stages) {
            if (it >= 1) ok = mbar_wait(&bar[(it - 1) % NS], ((it - 1) / NS) & 1);
            if (ok) issue(nxt);
        }
        cp_async_commit();
    }
    cp_async_wait<0>();
    // the last commit covers every earlier MMA of this thread; it is waited
    // for on the error path too, before the tensor memory is freed
    if (issued > 0 && !mbar_wait(&bar[(issued - 1) % NS], ((issued - 1) / NS) & 1)) ok = false;
    ok = __syncthreads_and(ok && issued == n_stages);
    tc_fence_after();

    if (ok) {
        const int q = warp & 3, half = warp >> 2;
        const int row_i = q * 32 + lane;
        const long long v = m0 + row_i;
        for (int c0 = half * 8; c0 < N; c0 += 16) {
            float f[8];
            tmem_ld8(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, f);
            if (v < P.n_vox) conv_store(P, v, c0, N, f);
        }
    } else if (tid == 0) {
        atomicOr(&g_status, 1u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, tmem_cols(N));
}

// ---------------------------------------------------------------------------
// forward / backward-data convolution from a shared-memory halo
// ---------------------------------------------------------------------------

// For a tile of 16 (y) x 8 (x) output voxels at one z, the input halo of
// 3 x 18 x 10 voxels is loaded into shared memory once, 8-channel chunk
// planes of 540 voxels x 16 bytes.  Each tap's A operand is then the same
// halo under a shifted descriptor start: the 8 rows of a core matrix are 8
// consecutive x voxels (16 bytes apart, 128 contiguous bytes), the 16 row
// groups are the tile's y rows (SBO = one halo row, 160 bytes), the two
// 8-channel halves of a K = 16 step are two chunk planes (LBO = 8640
// bytes) -- a valid K-major no-swizzle operand for every tap, so the 27
// taps' MMAs need no gather.  The packed weights are chunk-major over
// K = 27 x cin, so tap t's chunk pair (2j, 2j + 1) is the B operand at
// chunk t * cin / 8 + 2j.  Used where the halo and all weights fit in
// shared memory (cin, N <= 48) and the tile divides the volume (H % 16,
// W % 8).
constexpr int HALO_Y = 18, HALO_X = 10, HALO_V = 3 * HALO_Y * HALO_X;

__host__ __device__ constexpr uint32_t halo_smem_bytes(int n, int cin) {
    return (uint32_t)(cin / 8) * HALO_V * 16 + (uint32_t)((27 * cin + KS - 1) / KS) * 8 * n * 16;
}

template <int N>
__global__ void __launch_bounds__(THREADS) conv_halo_kernel(const ConvP P) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Src& S = P.src;
    const int cin = S.ca + S.cb, c8n = cin / 8;
    const int tiles_x = S.W / 8, tiles_y = S.H / 16;
    int t = blockIdx.x;
    const int x0 = (t % tiles_x) * 8;
    t /= tiles_x;
    const int y0 = (t % tiles_y) * 16;
    t /= tiles_y;
    const int z = t % S.D, n = t / S.D;
    const uint32_t halo_bytes = (uint32_t)c8n * HALO_V * 16;
    const int w_chunks = ((27 * cin + KS - 1) / KS) * 8 * N;

    if (warp == 0) tmem_alloc(&s_tmem, tmem_cols(N));
    if (tid == 0) {
        mbar_init(&bar, 1);
        mbar_init_fence();
    }
    const uint32_t sbase = smem_u32(smem), swt = sbase + halo_bytes;
    // halo: chunk c8, voxel hv = (hz * 18 + hy) * 10 + hx
    for (int i = tid; i < c8n * HALO_V; i += THREADS) {
        const int c8 = i / HALO_V, hv = i - c8 * HALO_V;
        const int hz = hv / (HALO_Y * HALO_X), hy = (hv / HALO_X) % HALO_Y, hx = hv % HALO_X;
        const int zz = z + hz - 1, yy = y0 + hy - 1, xx = x0 + hx - 1;
        const int ch = c8 * 8;
        uint32_t bytes = 0;
        const void* src = S.a;
        if ((unsigned)zz < (unsigned)S.D && (unsigned)yy < (unsigned)S.H && (unsigned)xx < (unsigned)S.W) {
            bytes = 16;
            if (ch < S.ca) {
                src = S.a + ((((size_t)n * S.D + zz) * S.H + yy) * S.W + xx) * S.ca + ch;
            } else {
                const size_t cv = (((size_t)n * (S.D >> 1) + (zz >> 1)) * (S.H >> 1) + (yy >> 1)) * (S.W >> 1) + (xx >> 1);
                src = S.b + cv * S.cb + (ch - S.ca);
            }
        }
        cp_async16(sbase + (uint32_t)i * 16, src, bytes);
    }
    for (int i = tid; i < w_chunks; i += THREADS) cp_async16(swt + (uint32_t)i * 16, P.w + (size_t)i * 8, 16u);
    cp_async_commit();
    cp_async_wait<0>();
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    constexpr uint32_t IDESC = idesc_bf16(TILE_M, N, 0, 0);
    if (tid == 0) {
        for (int tap = 0; tap < 27; ++tap) {
            const uint32_t off = (uint32_t)(((tap / 9) * HALO_Y + (tap / 3) % 3) * HALO_X + tap % 3) * 16;
            for (int j = 0; j < c8n / 2; ++j) {
                uint64_t ad = smem_desc(sbase + (uint32_t)(2 * j) * HALO_V * 16 + off, HALO_V * 16, HALO_X * 16);
                uint64_t bd = smem_desc(swt + (uint32_t)(tap * c8n + 2 * j) * N * 16, N * 16, 128);
                mma_bf16(tmem, ad, bd, IDESC, (tap > 0 || j > 0) ? 1u : 0u);
            }
        }
        mma_commit(&bar);
    }
    const bool ok = __syncthreads_and(mbar_wait(&bar, 0));
    tc_fence_after();
    if (ok) {
        const int q = warp & 3, half = warp >> 2;
        const int m = q * 32 + lane;
        const long long v = (((long long)n * S.D + z) * S.H + y0 + (m >> 3)) * S.W + x0 + (m & 7);
        for (int c0 = half * 8; c0 < N; c0 += 16) {
            float f[8];
            tmem_ld8(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, f);
            conv_store(P, v, c0, N, f);
        }
    } else if (tid == 0) {
        atomicOr(&g_status, 1u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, tmem_cols(N));
}

// ---------------------------------------------------------------------------
// forward / backward-data convolution streaming z-planes through a halo ring
// ---------------------------------------------------------------------------

// A persistent version of the halo kernel.  A work item is a column of
// output tiles (16 y x 8 x, one z each) over ZSEG consecutive z of one
// volume; the CTA keeps the layer's packed weights in shared memory for all
// its items and a ring of four 18 x 10 halo planes, so each input plane is
// loaded once per column instead of three times, and the weights once per
// CTA instead of once per tile.  Per output plane z: one thread issues the
// 27 x cin/16 MMAs of z into one of two tensor-memory accumulators, then
// all threads wait for the MMAs of z - 1, copy plane z + 2 into the ring
// slot that plane z - 2 held, and store z - 1's outputs from the other
// accumulator -- loads, MMAs and epilogue of neighbouring planes overlap.
// The ring slot of plane p of an item starting at zs is (p - zs + 1) & 3;
// the operand descriptors are the halo kernel's (8 x voxels per core
// matrix row, SBO one halo row, LBO one 8-channel plane).  The issuing
// thread starts plane z's MMAs once those of z - 1 are done, so that its
// issue overlaps the other warps' copies and epilogue.
constexpr int ZSEG = 16;
constexpr int RING_V = HALO_Y * HALO_X;               // voxels of one halo plane

__host__ __device__ constexpr uint32_t stream_acc_cols(int n) { return n <= 32 ? 32u : 64u; }
__host__ __device__ constexpr uint32_t stream_tmem_cols(int n) { return 2u * stream_acc_cols(n); }
__host__ __device__ constexpr uint32_t stream_smem_bytes(int n, int cin) {
    return 4u * (uint32_t)(cin / 8) * RING_V * 16 + (uint32_t)((27 * cin + KS - 1) / KS) * 8 * n * 16;
}

template <int N>
__global__ void __launch_bounds__(THREADS) conv_stream_kernel(const ConvP P, int n_items) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ uint64_t bar[2];
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Src& S = P.src;
    const int cin = S.ca + S.cb, c8n = cin / 8;
    // edge tiles reach past the volume: their halo reads zeros there and
    // their outputs outside it are not stored
    const int tiles_x = (S.W + 7) / 8, tiles_y = (S.H + 15) / 16, n_seg = (S.D + ZSEG - 1) / ZSEG;
    const uint32_t ring_bytes = 4u * (uint32_t)c8n * RING_V * 16;
    const int w_chunks = ((27 * cin + KS - 1) / KS) * 8 * N;
    constexpr uint32_t ACC = stream_acc_cols(N);

    if (warp == 0) tmem_alloc(&s_tmem, stream_tmem_cols(N));
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init_fence();
    }
    const uint32_t sbase = smem_u32(smem), swt = sbase + ring_bytes;
    for (int i = tid; i < w_chunks; i += THREADS) cp_async16(swt + (uint32_t)i * 16, P.w + (size_t)i * 8, 16u);
    cp_async_commit();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    constexpr uint32_t IDESC = idesc_bf16(TILE_M, N, 0, 0);
    const int q = warp & 3, half = warp >> 2;

    // copies of input plane zz (zero outside the volume) of column (n, y0, x0) into ring slot
    auto load_plane = [&](int n, int y0, int x0, int zz, int slot) {
        const uint32_t base = sbase + (uint32_t)slot * c8n * RING_V * 16;
        for (int i = tid; i < c8n * RING_V; i += THREADS) {
            const int c8 = i / RING_V, hv = i - c8 * RING_V;
            const int yy = y0 + hv / HALO_X - 1, xx = x0 + hv % HALO_X - 1;
            const int ch = c8 * 8;
            uint32_t bytes = 0;
            const void* src = S.a;
            if ((unsigned)zz < (unsigned)S.D && (unsigned)yy < (unsigned)S.H && (unsigned)xx < (unsigned)S.W) {
                bytes = 16;
                if (ch < S.ca) {
                    src = S.a + ((((size_t)n * S.D + zz) * S.H + yy) * S.W + xx) * S.ca + ch;
                } else {
                    const size_t cv =
                        (((size_t)n * (S.D >> 1) + (zz >> 1)) * (S.H >> 1) + (yy >> 1)) * (S.W >> 1) + (xx >> 1);
                    src = S.b + cv * S.cb + (ch - S.ca);
                }
            }
            cp_async16(base + (uint32_t)(c8 * RING_V + hv) * 16, src, bytes);
        }
    };
    // outputs of plane z of the column from the accumulator of commit k
    auto store_plane = [&](int n, int y0, int x0, int z, uint32_t k) {
        const uint32_t acc = tmem + (k & 1u) * ACC;
        const int m = q * 32 + lane;
        const int y = y0 + (m >> 3), x = x0 + (m & 7);
        const long long v = (((long long)n * S.D + z) * S.H + y) * S.W + x;
        for (int c0 = half * 8; c0 < N; c0 += 16) {
            float f[8];
            tmem_ld8(acc + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, f);   // every lane: warp-collective
            if (y < S.H && x < S.W) conv_store(P, v, c0, N, f);
        }
    };

    bool ok = true;
    uint32_t commits = 0;                      // MMA groups committed by this CTA (bar[k & 1], phase k >> 1)
    for (int item = blockIdx.x; item < n_items && ok; item += gridDim.x) {
        int t = item;
        const int seg = t % n_seg;
        t /= n_seg;
        const int x0 = (t % tiles_x) * 8;
        t /= tiles_x;
        const int y0 = (t % tiles_y) * 16;
        const int n = t / tiles_y;
        const int zs = seg * ZSEG, ze = min(zs + ZSEG, S.D);
        for (int r = 0; r < 3; ++r) load_plane(n, y0, x0, zs - 1 + r, r);
        cp_async_commit();
        cp_async_wait<0>();
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        for (int z = zs; z < ze; ++z) {
            const int i = z - zs;
            if (i > 0) {
                // the MMAs of z - 1: their accumulator is ready and plane z - 2 is free
                const uint32_t kp = commits - 1;
                const bool w = mbar_wait(&bar[kp & 1u], (kp >> 1) & 1u);
                ok = __syncthreads_and(ok && w) != 0;      // uniform before the warp-collective loads
                tc_fence_after();
                if (!ok) break;
            }
            const uint32_t k = commits++;
            if (tid == 0) {
                // the 27 x cin/16 MMAs of plane z; the descriptors differ from
                // the first one by their start addresses only (in 16-byte units)
                const uint32_t acc = tmem + (k & 1u) * ACC;
                const uint64_t a0 = smem_desc(sbase, RING_V * 16, HALO_X * 16);
                const uint64_t b0 = smem_desc(swt, N * 16, 128);
                const uint32_t slot16 = (uint32_t)c8n * RING_V;
                const uint32_t so[3] = {(uint32_t)(i & 3) * slot16, (uint32_t)((i + 1) & 3) * slot16,
                                        (uint32_t)((i + 2) & 3) * slot16};
#pragma unroll
                for (int tap = 0; tap < 27; ++tap) {
                    const uint32_t ta = so[tap / 9] + (uint32_t)(((tap / 3) % 3) * HALO_X + tap % 3);
                    for (int j = 0; j < c8n / 2; ++j)
                        mma_bf16(acc, a0 + ta + (uint32_t)(2 * j * RING_V), b0 + (uint32_t)((tap * c8n + 2 * j) * N),
                                 IDESC, (tap > 0 || j > 0) ? 1u : 0u);
                }
                mma_commit(&bar[k & 1u]);
            }
            if (z + 2 <= ze) load_plane(n, y0, x0, z + 2, (i + 3) & 3);
            cp_async_commit();
            if (i > 0) store_plane(n, y0, x0, z - 1, k - 1);
            cp_async_wait<0>();
            fence_proxy_async();
            tc_fence_before();
            ok = __syncthreads_and(ok) != 0;
            tc_fence_after();
            if (!ok) break;
        }
        if (!ok) break;
        // the last plane of the item
        const uint32_t k = commits - 1;
        const bool w = mbar_wait(&bar[k & 1u], (k >> 1) & 1u);
        ok = __syncthreads_and(w) != 0;
        tc_fence_after();
        if (!ok) break;
        store_plane(n, y0, x0, ze - 1, k);
        tc_fence_before();
        ok = __syncthreads_and(ok) != 0;
        tc_fence_after();
    }
    if (!ok) {
        // every committed MMA group has finished (or its wait ran out) before the memory is freed
        if (commits > 0) mbar_wait(&bar[(commits - 1) & 1u], ((commits - 1) >> 1) & 1u);
        if (tid == 0) atomicOr(&g_status, 1u);
    }
    cp_async_wait<0>();
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, stream_tmem_cols(N));
}

// ---------------------------------------------------------------------------
// the same streaming convolution with warp roles and no block-wide barriers
// ---------------------------------------------------------------------------

// The work unit is conv_stream_kernel's (output planes of one 16 x 8 column,
// fed by a ring of halo planes, the packed weights resident), but:
//  - each CTA takes one contiguous range of the (column, plane) sequence,
//    T / gridDim.x planes, so that every CTA has the same work to within one
//    plane; the range is cut into segments at column ends;
//  - the ring holds `ring` planes (4 .. WS_RING_MAX), so that the copies run
//    up to ring - 3 planes ahead of the MMAs;
//  - the CTA's warps take fixed roles that hand work to each other through
//    mbarriers instead of meeting at __syncthreads:
//      warp 0, one thread: waits for the three input planes of output plane
//        z and for a free accumulator, issues the 27 x cin/16 MMAs, commits
//        to "accumulator full" and to "plane free" of the planes z's MMAs
//        read last;
//      warps 1-3: copy input planes into the ring as slots come free (each
//        thread waits for its own copies, fences them for the tensor core
//        and arrives on the slot's "plane full");
//      warps 4-7: one output row per thread (the four warps are the four
//        tensor-memory lane quarters), read an accumulator, store it and
//        arrive on "accumulator free".
// Plane L of the CTA's sequence (the planes zs - 1 .. ze of each segment in
// turn) lives in ring slot L % ring; the MMAs of output plane z read planes
// base + i .. base + i + 2 (i = z - zs, base the segment's first plane); z
// is the last reader of plane base + i, and of the segment's last two
// planes when z is its last output.
constexpr int WS_RING_MAX = 12;
constexpr int WS_LOADERS = 96;              // warps 1-3

__host__ __device__ constexpr uint32_t ws_smem_bytes(int n, int cin, int ring) {
    return (uint32_t)ring * (uint32_t)(cin / 8) * RING_V * 16 + (uint32_t)((27 * cin + KS - 1) / KS) * 8 * n * 16;
}

// Segment of the CTA's plane range that starts at sequence position g (g <
// end): column (n, y0, x0), output planes [zs, ze).
struct WsSeg {
    int n, y0, x0, zs, ze;
};
__device__ __forceinline__ WsSeg ws_segment(const Src& S, long long g, long long end, int tiles_x, int tiles_y) {
    WsSeg q;
    const long long col = g / S.D;
    q.zs = (int)(g - col * S.D);
    q.ze = (int)min((long long)S.D, (long long)q.zs + (end - g));
    q.x0 = (int)(col % tiles_x) * 8;
    const long long r = col / tiles_x;
    q.y0 = (int)(r % tiles_y) * 16;
    q.n = (int)(r / tiles_y);
    return q;
}

template <int N>
__global__ void __launch_bounds__(THREADS, 4) conv_ws_kernel(const ConvP P, int ring) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ uint64_t full[WS_RING_MAX], empty[WS_RING_MAX], accf[2], acce[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Src& S = P.src;
    const int cin = S.ca + S.cb, c8n = cin / 8;
    const int tiles_x = (S.W + 7) / 8, tiles_y = (S.H + 15) / 16;
    const long long total = (long long)S.B * tiles_y * tiles_x * S.D;
    const long long g_begin = total * blockIdx.x / gridDim.x, g_end = total * (blockIdx.x + 1) / gridDim.x;
    const uint32_t R = (uint32_t)ring;
    const uint32_t slot16 = (uint32_t)c8n * RING_V;           // one ring slot, 16-byte units
    const uint32_t ring_bytes = R * slot16 * 16;
    const int w_chunks = ((27 * cin + KS - 1) / KS) * 8 * N;
    constexpr uint32_t ACC = stream_acc_cols(N);
    volatile int* fail = &s_fail;

    if (warp == 0) tmem_alloc(&s_tmem, stream_tmem_cols(N));
    if (tid == 0) {
        for (uint32_t r = 0; r < R; ++r) {
            mbar_init(&full[r], WS_LOADERS);
            mbar_init(&empty[r], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&accf[b], 1);
            mbar_init(&acce[b], 128);
        }
        s_fail = 0;
        mbar_init_fence();
    }
    const uint32_t sbase = smem_u32(smem), swt = sbase + ring_bytes;
    for (int i = tid; i < w_chunks; i += THREADS) cp_async16(swt + (uint32_t)i * 16, P.w + (size_t)i * 8, 16u);
    cp_async_commit();
    cp_async_wait<0>();
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;

    if (warp >= 1 && warp <= 3) {
        // ---- loaders ----
        const int lt = tid - 32;
        uint32_t L = 0;                       // planes issued by this CTA
        bool pending = false;                 // plane L - 1 issued but not yet published
        for (long long g = g_begin; g < g_end && !*fail;) {
            const WsSeg q = ws_segment(S, g, g_end, tiles_x, tiles_y);
            g += q.ze - q.zs;
            for (int zz = q.zs - 1; zz <= q.ze && !*fail; ++zz, ++L) {
                const uint32_t slot = L % R;
                if (L >= R) {
                    const uint32_t par = ((L / R) - 1) & 1u;
                    if (!mbar_try_wait(&empty[slot], par)) {
                        // the slot is still read: publish the previous plane first
                        if (pending) {
                            cp_async_wait<0>();
                            fence_proxy_async();
                            mbar_arrive(&full[(L - 1) % R]);
                            pending = false;
                        }
                        if (!mbar_wait_or_fail(&empty[slot], par, fail)) break;
                    }
                }
                const uint32_t base = sbase + slot * slot16 * 16;
                for (int i = lt; i < c8n * RING_V; i += WS_LOADERS) {
                    const int c8 = i / RING_V, hv = i - c8 * RING_V;
                    const int yy = q.y0 + hv / HALO_X - 1, xx = q.x0 + hv % HALO_X - 1;
                    const int ch = c8 * 8;
                    uint32_t bytes = 0;
                    const void* src = S.a;
                    if ((unsigned)zz < (unsigned)S.D && (unsigned)yy < (unsigned)S.H && (unsigned)xx < (unsigned)S.W) {
                        bytes = 16;
                        if (ch < S.ca) {
                            src = S.a + ((((size_t)q.n * S.D + zz) * S.H + yy) * S.W + xx) * S.ca + ch;
                        } else {
                            const size_t cv = (((size_t)q.n * (S.D >> 1) + (zz >> 1)) * (S.H >> 1) + (yy >> 1)) *
                                                  (S.W >> 1) + (xx >> 1);
                            src = S.b + cv * S.cb + (ch - S.ca);
                        }
                    }
                    cp_async16(base + (uint32_t)i * 16, src, bytes);
                }
                cp_async_commit();
                // the previous plane's copies of this thread have landed: publish them
                if (pending) {
                    cp_async_wait<1>();
                    fence_proxy_async();
                    mbar_arrive(&full[(L - 1) % R]);
                }
                pending = true;
            }
        }
        cp_async_wait<0>();
        fence_proxy_async();
        if (pending && !*fail) mbar_arrive(&full[(L - 1) % R]);
    } else if (warp == 0 && lane == 0) {
        // ---- MMA issuer ----
        uint32_t K = 0, waited = 0, base = 0;     // output planes issued, input planes seen full, segment's first plane
        const uint64_t a0 = smem_desc(sbase, RING_V * 16, HALO_X * 16);
        const uint64_t b0 = smem_desc(swt, N * 16, 128);
        constexpr uint32_t IDESC = idesc_bf16(TILE_M, N, 0, 0);
        for (long long g = g_begin; g < g_end && !*fail;) {
            const WsSeg q = ws_segment(S, g, g_end, tiles_x, tiles_y);
            g += q.ze - q.zs;
            for (int z = q.zs; z < q.ze && !*fail; ++z, ++K) {
                const uint32_t p0 = base + (uint32_t)(z - q.zs);          // plane z - 1
                bool ok = true;
                while (ok && waited <= p0 + 2) {
                    ok = mbar_wait_or_fail(&full[waited % R], (waited / R) & 1u, fail);
                    ++waited;
                }
                if (ok && K >= 2) ok = mbar_wait_or_fail(&acce[K & 1u], ((K >> 1) - 1) & 1u, fail);
                if (!ok) break;
                tc_fence_after();
                const uint32_t acc = tmem + (K & 1u) * ACC;
                const uint32_t s0 = (p0 % R) * slot16, s1 = ((p0 + 1) % R) * slot16, s2 = ((p0 + 2) % R) * slot16;
                for (int dz = 0; dz < 3; ++dz) {
                    const uint32_t so = dz == 0 ? s0 : (dz == 1 ? s1 : s2);
#pragma unroll
                    for (int t = 0; t < 9; ++t) {
                        const int tap = dz * 9 + t;
                        const uint32_t ta = so + (uint32_t)((t / 3) * HALO_X + t % 3);
                        for (int j = 0; j < c8n / 2; ++j)
                            mma_bf16(acc, a0 + ta + (uint32_t)(2 * j * RING_V),
                                     b0 + (uint32_t)((tap * c8n + 2 * j) * N), IDESC, (tap > 0 || j > 0) ? 1u : 0u);
                    }
                }
                mma_commit(&accf[K & 1u]);
                mma_commit(&empty[p0 % R]);
                if (z == q.ze - 1) {
                    mma_commit(&empty[(p0 + 1) % R]);
                    mma_commit(&empty[(p0 + 2) % R]);
                }
            }
            base += (uint32_t)(q.ze - q.zs) + 2;
        }
        // every issued MMA has finished before the tensor memory can be freed
        if (K > 0) mbar_wait(&accf[(K - 1) & 1u], ((K - 1) >> 1) & 1u);
    } else if (warp >= 4) {
        // ---- epilogue: row m of the tile, lane quarter warp - 4 ----
        const int qw = warp - 4, m = qw * 32 + lane;
        uint32_t K = 0;
        for (long long g = g_begin; g < g_end && !*fail;) {
            const WsSeg q = ws_segment(S, g, g_end, tiles_x, tiles_y);
            g += q.ze - q.zs;
            const int y = q.y0 + (m >> 3), x = q.x0 + (m & 7);
            for (int z = q.zs; z < q.ze; ++z, ++K) {
                // one waiter per warp keeps the warp-collective loads uniform
                int w = 1;
                if (lane == 0) w = mbar_wait_or_fail(&accf[K & 1u], (K >> 1) & 1u, fail) ? 1 : 0;
                if (!__shfl_sync(0xffffffffu, w, 0)) break;
                tc_fence_after();
                const uint32_t acc = tmem + (K & 1u) * ACC + ((uint32_t)(qw * 32) << 16);
                const long long v = (((long long)q.n * S.D + z) * S.H + y) * S.W + x;
#pragma unroll
                for (int c0 = 0; c0 < N; c0 += 8) {
                    float f[8];
                    tmem_ld8(acc + (uint32_t)c0, f);
                    if (y < S.H && x < S.W) conv_store(P, v, c0, N, f);
                }
                tc_fence_before();
                mbar_arrive(&acce[K & 1u]);
            }
        }
    }
    __syncthreads();
    if (tid == 0 && s_fail) atomicOr(&g_status, 1u);
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, stream_tmem_cols(N));
}

// ---------------------------------------------------------------------------
// plane-stationary streaming convolution (16 or 32 output channels)
// ---------------------------------------------------------------------------

// A tcgen05.mma that accumulates into the accumulator of the previous one
// waits for it: a chain of MMAs on one accumulator runs at one MMA per
// ~125 cycles (A in shared memory) whatever N is, so 16 or 32 output
// channels per MMA leave the tensor core mostly idle.  Here each input
// plane p is read by ONE chain of 9 x cin/16 MMAs (the in-plane taps dy,
// dx) against the three weight planes dz stacked along N (N = 3 x cout):
//     D_p[m][dz * cout + co] = sum_{dy, dx, ci} W[dz, dy, dx][co][ci] x_p(m + (dy, dx))[ci]
// and output plane z is D_{z-1}[.., 0 | ..] + D_z[.., 1 | ..] + D_{z+1}[.., 2 | ..],
// summed in FP32 by the epilogue from three tensor-memory regions.  A is
// read a third as often as by the output-stationary kernels, and N is
// three times wider.  Q = 5 regions of 3 x cout columns: the MMAs of
// plane p + 1 and p + 2 overlap the epilogue of output p - 1.
// Work split, ring of halo planes, warp roles and loader as conv_ws_kernel;
// the barriers are: full / empty per ring slot (one MMA group reads each
// plane), rfull per region (the plane's MMAs are done) and rfree per region
// (the last output that reads the region, z + 1 for D_z, is stored).
// Issue groups: the MMA thread takes G consecutive planes at once and
// interleaves their chains tap by tap, so that G independent accumulator
// chains are in flight per CTA (one per plane); the CTA then holds
// 2 G + 2 regions (4 for G = 1).
// Channel passes: the kernel reads input channel groups [c8_lo, c8_hi) (8
// channels each) and the matching weight rows only, so that layers whose
// weights do not fit shared memory run as several passes: every pass but
// the last adds into an FP32 partial sum [v][NO] (part_out), the last adds
// the partial (part_in) before bias, ReLU, mask and the BF16 store.
// Output slices: a launch computes output channels [co_lo, co_lo + NO) of
// a layer with more (64 output channels: two slices of 32).
constexpr int PS_REGIONS_MAX = 8;
constexpr int PS_GROUP_MAX = 3;

// tensor-memory columns of one region: 3 x cout
__host__ __device__ constexpr uint32_t ps_region_cols(int n) { return 3u * (uint32_t)n; }
// regions for issue groups of g planes: 5 for g = 1 (plane L's MMAs need
// the region of plane L - 5, released once plane L - 3's MMAs are done:
// the issuing thread runs two planes ahead of the epilogue), else 2 g + 2;
// columns allocated
__host__ __device__ constexpr int ps_regions(int g) { return g <= 1 ? 5 : 2 * g + 2; }
__host__ __device__ constexpr uint32_t ps_tmem_cols(int n, int g) {
    return (uint32_t)ps_regions(g) * ps_region_cols(n) <= 256u ? 256u : 512u;
}
__host__ __device__ constexpr uint32_t ps_weight_bytes(int n, int c8p) { return 9u * (uint32_t)c8p * 3u * n * 16u; }
__host__ __device__ constexpr uint32_t ps_smem_bytes(int n, int c8p, int ring) {
    return (uint32_t)ring * (uint32_t)c8p * RING_V * 16 + ps_weight_bytes(n, c8p);
}

// next index of a ring of n entries, flipping the phase bit on wrap-around
__device__ __forceinline__ void ring_next(uint32_t& i, uint32_t& phase, uint32_t n) {
    if (++i == n) {
        i = 0;
        phase ^= 1u;
    }
}

struct PsPass {
    int c8_lo, c8_hi;          // input channel groups of this pass
    int co_lo, n_out;          // output channels [co_lo, co_lo + NO) of the layer's n_out
    const float* part_in;      // FP32 partial sums [v][NO] to add, or null
    float* part_out;           // FP32 sums [v][NO] out (no bias / ReLU / BF16), or null
};

template <int NO, int G>
__global__ void __launch_bounds__(THREADS, 1) conv_ps_kernel(const ConvP P, const PsPass Q, int ring) {
    constexpr int NP = 3 * NO;                                // MMA N: the three dz weight planes
    constexpr uint32_t RC = ps_region_cols(NO);
    constexpr uint32_t NQ = (uint32_t)ps_regions(G), TCOLS = ps_tmem_cols(NO, G);
    static_assert(NQ <= PS_REGIONS_MAX && NQ * RC <= 512, "issue group too large for the tensor memory");
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ uint64_t full[WS_RING_MAX], empty[WS_RING_MAX], rfull[PS_REGIONS_MAX], rfree[PS_REGIONS_MAX];
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Src& S = P.src;
    const int c8n = (S.ca + S.cb) / 8, c8p = Q.c8_hi - Q.c8_lo;
    const int tiles_x = (S.W + 7) / 8, tiles_y = (S.H + 15) / 16;
    const long long total = (long long)S.B * tiles_y * tiles_x * S.D;
    const long long g_begin = total * blockIdx.x / gridDim.x, g_end = total * (blockIdx.x + 1) / gridDim.x;
    const uint32_t R = (uint32_t)ring;
    const uint32_t slot16 = (uint32_t)c8p * RING_V;           // one ring slot, 16-byte units
    volatile int* fail = &s_fail;

    if (warp == 0) tmem_alloc(&s_tmem, TCOLS);
    if (tid == 0) {
        for (uint32_t r = 0; r < R; ++r) {
            mbar_init(&full[r], WS_LOADERS);
            mbar_init(&empty[r], 1);
        }
        for (uint32_t r = 0; r < NQ; ++r) {
            mbar_init(&rfull[r], 1);
            mbar_init(&rfree[r], 128);
        }
        s_fail = 0;
        mbar_init_fence();
    }
    // weights: packed chunk (tap * c8n + c8, co_lo + co) -> (t9 * c8p + c8 - c8_lo, dz * NO + co)
    const uint32_t sbase = smem_u32(smem), swt = sbase + R * slot16 * 16;
    for (int i = tid; i < 9 * c8p * NP; i += THREADS) {
        const int r = i % NP, g = i / NP;
        const int t9 = g / c8p, c8 = Q.c8_lo + g % c8p, dz = r / NO, co = r % NO;
        const int src = ((dz * 9 + t9) * c8n + c8) * Q.n_out + Q.co_lo + co;
        cp_async16(swt + (uint32_t)i * 16, P.w + (size_t)src * 8, 16u);
    }
    cp_async_commit();
    cp_async_wait<0>();
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;

    if (warp >= 1 && warp <= 3) {
        // ---- loaders: planes zs - 1 .. ze of each segment, channel groups of the pass ----
        // Each thread's copies of a plane arrive on the slot's "full" barrier
        // when they land, so the loaders never wait for their own copies:
        // as many planes are in flight as the ring has free slots.
        const int lt = tid - 32;
        uint32_t L = 0, slot = 0, ph = 0;             // plane, its ring slot and the slot's phase
        for (long long g = g_begin; g < g_end && !*fail;) {
            const WsSeg q = ws_segment(S, g, g_end, tiles_x, tiles_y);
            g += q.ze - q.zs;
            for (int zz = q.zs - 1; zz <= q.ze && !*fail; ++zz, ++L, ring_next(slot, ph, R)) {
                if (L >= R && !mbar_wait_or_fail(&empty[slot], ph ^ 1u, fail)) break;
                const uint32_t base = sbase + slot * slot16 * 16;
                for (int i = lt; i < c8p * RING_V; i += WS_LOADERS) {
                    const int c8 = i / RING_V, hv = i - c8 * RING_V;
                    const int yy = q.y0 + hv / HALO_X - 1, xx = q.x0 + hv % HALO_X - 1;
                    const int ch = (Q.c8_lo + c8) * 8;
                    uint32_t bytes = 0;
                    const void* src = S.a;
                    if ((unsigned)zz < (unsigned)S.D && (unsigned)yy < (unsigned)S.H && (unsigned)xx < (unsigned)S.W) {
                        bytes = 16;
                        if (ch < S.ca) {
                            src = S.a + ((((size_t)q.n * S.D + zz) * S.H + yy) * S.W + xx) * S.ca + ch;
                        } else {
                            const size_t cv = (((size_t)q.n * (S.D >> 1) + (zz >> 1)) * (S.H >> 1) + (yy >> 1)) *
                                                  (S.W >> 1) + (xx >> 1);
                            src = S.b + cv * S.cb + (ch - S.ca);
                        }
                    }
                    cp_async16_cg(base + (uint32_t)i * 16, src, bytes);
                }
                cp_async_arrive_noinc(&full[slot]);
            }
        }
        cp_async_wait<0>();
    } else if (warp == 0 && lane == 0) {
        // ---- MMA issuer: per input plane one chain of 9 x c8p / 2 MMAs; the chains of a
        // group of planes are issued tap by tap in turn ----
        const uint64_t a0 = smem_desc(sbase, RING_V * 16, HALO_X * 16);
        const uint64_t b0 = smem_desc(swt, NP * 16, 128);
        constexpr uint32_t IDESC = idesc_bf16(TILE_M, NP, 0, 0);
        uint32_t n_planes = 0;                       // planes of the CTA's sequence: each segment's zs - 1 .. ze
        for (long long g = g_begin; g < g_end;) {
            const WsSeg q = ws_segment(S, g, g_end, tiles_x, tiles_y);
            g += q.ze - q.zs;
            n_planes += (uint32_t)(q.ze - q.zs) + 2;
        }
        // plane L's ring slot and region with their phases, advanced without divisions
        uint32_t L = 0, fs = 0, fph = 0, rs = 0, rph = 0;
        bool ok = true;
        while (L < n_planes && ok && !*fail) {
            const uint32_t gn = min((uint32_t)G, n_planes - L);      // G but for the CTA's last group
            uint32_t d[G], so[G], fsk[G], rsk[G];
            {
                uint32_t f = fs, fp = fph, r = rs, rp = rph;
#pragma unroll
                for (int k = 0; k < G; ++k) {
                    fsk[k] = f;
                    rsk[k] = r;
                    d[k] = tmem + r * RC;
                    so[k] = f * slot16;
                    if (G == 1 || (uint32_t)k < gn) {
                        if (ok) ok = mbar_wait_or_fail(&full[f], fp, fail);
                        if (ok && L + k >= NQ) ok = mbar_wait_or_fail(&rfree[r], rp ^ 1u, fail);
                    }
                    ring_next(f, fp, R);
                    ring_next(r, rp, NQ);
                }
            }
            if (!ok) break;
            fence_proxy_async();              // the loaders' copies, seen through the barrier, to the tensor core
            tc_fence_after();
#pragma unroll
            for (int t9 = 0; t9 < 9; ++t9) {
                const uint32_t ta = (uint32_t)((t9 / 3) * HALO_X + t9 % 3);
                for (int j = 0; j < c8p / 2; ++j) {
                    const uint64_t bd = b0 + (uint32_t)((t9 * c8p + 2 * j) * NP);
                    const uint32_t acc = (t9 > 0 || j > 0) ? 1u : 0u;
#pragma unroll
                    for (int k = 0; k < G; ++k)
                        if (G == 1 || (uint32_t)k < gn)
                            mma_bf16(d[k], a0 + so[k] + ta + (uint32_t)(2 * j * RING_V), bd, IDESC, acc);
                }
            }
#pragma unroll
            for (int k = 0; k < G; ++k)
                if (G == 1 || (uint32_t)k < gn) {
                    mma_commit(&rfull[rsk[k]]);
                    mma_commit(&empty[fsk[k]]);
                }
            for (uint32_t k = 0; k < gn; ++k) {
                ring_next(fs, fph, R);
                ring_next(rs, rph, NQ);
            }
            L += gn;
        }
        // every issued MMA has finished before the tensor memory can be freed: plane L - 1's phase
        if (L > 0) mbar_wait(&rfull[rs == 0 ? NQ - 1 : rs - 1], rs == 0 ? rph ^ 1u : rph);
    } else if (warp >= 4) {
        // ---- epilogue: output z = D_{z-1}[dz 0] + D_z[dz 1] + D_{z+1}[dz 2]; row m, lane quarter warp - 4 ----
        const int qw = warp - 4, m = qw * 32 + lane;
        const uint32_t lq = (uint32_t)(qw * 32) << 16;
        // region and phase of plane z + 1, and the regions of planes z and z - 1
        uint32_t r1 = 0, ph1 = 0;
        ring_next(r1, ph1, NQ);
        ring_next(r1, ph1, NQ);                                // the first output reads planes 0, 1, 2
        for (long long g = g_begin; g < g_end && !*fail;) {
            const WsSeg q = ws_segment(S, g, g_end, tiles_x, tiles_y);
            g += q.ze - q.zs;
            const int y = q.y0 + (m >> 3), x = q.x0 + (m & 7);
            const bool in = y < S.H && x < S.W;
            bool ok = true;
            for (int z = q.zs; z < q.ze; ++z, ring_next(r1, ph1, NQ)) {
                const uint32_t r0i = r1 == 0 ? NQ - 1 : r1 - 1, rmi = r0i == 0 ? NQ - 1 : r0i - 1;
                int w = 1;
                if (lane == 0) w = mbar_wait_or_fail(&rfull[r1], ph1, fail) ? 1 : 0;
                if (!__shfl_sync(0xffffffffu, w, 0)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t rm = tmem + rmi * RC + lq;
                const uint32_t r0 = tmem + r0i * RC + NO + lq;
                const uint32_t rp = tmem + r1 * RC + 2 * NO + lq;
                const long long v = (((long long)q.n * S.D + z) * S.H + y) * S.W + x;
                // the head: x + b, then + w_j a_j in channel order (the head kernel's FP32 sequence)
                const bool head = NO == 16 && P.head && in;
                float hsum = head ? P.head_x[v] + __ldg(P.head + 16) : 0.0f;
                // the three regions' loads of 16 channels in flight together
#pragma unroll
                for (int c0 = 0; c0 < NO; c0 += 16) {
                    uint32_t u[6][8];
                    tmem_ld8_nw(rm + (uint32_t)c0, u[0]);
                    tmem_ld8_nw(r0 + (uint32_t)c0, u[1]);
                    tmem_ld8_nw(rp + (uint32_t)c0, u[2]);
                    tmem_ld8_nw(rm + (uint32_t)c0 + 8, u[3]);
                    tmem_ld8_nw(r0 + (uint32_t)c0 + 8, u[4]);
                    tmem_ld8_nw(rp + (uint32_t)c0 + 8, u[5]);
                    tmem_wait_ld();
                    if (!in) continue;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int c = c0 + 8 * h;
                        float f[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j)
                            f[j] = (__uint_as_float(u[3 * h][j]) + __uint_as_float(u[3 * h + 1][j])) +
                                   __uint_as_float(u[3 * h + 2][j]);
                        if (Q.part_in) {
                            const float4* pi = reinterpret_cast<const float4*>(Q.part_in + (size_t)v * NO + c);
                            const float4 u0 = __ldg(pi), u1 = __ldg(pi + 1);
                            f[0] += u0.x, f[1] += u0.y, f[2] += u0.z, f[3] += u0.w;
                            f[4] += u1.x, f[5] += u1.y, f[6] += u1.z, f[7] += u1.w;
                        }
                        if (Q.part_out) {
                            float4* po = reinterpret_cast<float4*>(Q.part_out + (size_t)v * NO + c);
                            po[0] = make_float4(f[0], f[1], f[2], f[3]);
                            po[1] = make_float4(f[4], f[5], f[6], f[7]);
                        } else {
                            conv_store(P, v, Q.co_lo + c, Q.n_out, f);
                            if (head) {
#pragma unroll
                                for (int j = 0; j < 8; ++j)
                                    hsum = fmaf(__ldg(P.head + c + j), __bfloat162float(__float2bfloat16_rn(f[j])),
                                                hsum);
                            }
                        }
                    }
                }
                if (head) P.head_out[v] = hsum;
                tc_fence_before();
                mbar_arrive(&rfree[rmi]);                               // plane z - 1: last reader done
                if (z == q.ze - 1) {
                    mbar_arrive(&rfree[r0i]);
                    mbar_arrive(&rfree[r1]);
                }
            }
            if (!ok) break;
            // the next segment's first output reads its planes 0 .. 2: two planes on
            ring_next(r1, ph1, NQ);
            ring_next(r1, ph1, NQ);
        }
    }
    __syncthreads();
    if (tid == 0 && s_fail) atomicOr(&g_status, 1u);
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, TCOLS);
}

// ---------------------------------------------------------------------------
// weight gradient: dW[tap][co][ci] += sum_v dz[v][co] * X[v + off(tap)][ci]
// ---------------------------------------------------------------------------

struct WgradP {
    Src src;
    const __nv_bfloat16* dz;     // [n_vox][N]
    long long n_vox;
    long long vox_per_cta;       // multiple of KSTAGE
    float* dw;                   // [27][N][cin], accumulated
};

__host__ __device__ constexpr int wgrad_stages(int n) { return n <= 64 ? 4 : 3; }
__host__ __device__ constexpr uint32_t wgrad_stage_bytes(int n) { return (uint32_t)(TILE_M + n) * KSTAGE * 2; }

// M = 128 rows (tap, ci) of 27 x cin, N = output channels, K = the CTA's
// voxel range in stages of KSTAGE voxels; both operands MN-major.  Each
// thread gathers one row group (8 channels of one tap) for four voxels of
// every stage.
template <int N>
__global__ void __launch_bounds__(THREADS) wgrad_kernel(const WgradP P) {
    constexpr int NS = wgrad_stages(N);
    constexpr uint32_t A_BYTES = TILE_M * KSTAGE * 2, STAGE = wgrad_stage_bytes(N);
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ uint64_t bar[NS];
    __shared__ uint32_t s_tmem;
    __shared__ VoxRec s_vox[NS][KSTAGE];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Src& S = P.src;
    const int cin = S.ca + S.cb;
    const int rows = 27 * cin;
    const int r0 = blockIdx.x * TILE_M;
    const long long v_begin = (long long)blockIdx.y * P.vox_per_cta;
    const long long v_end = v_begin + P.vox_per_cta < P.n_vox ? v_begin + P.vox_per_cta : P.n_vox;
    const int n_stages = v_end > v_begin ? (int)((v_end - v_begin + KSTAGE - 1) / KSTAGE) : 0;

    if (warp == 0) tmem_alloc(&s_tmem, tmem_cols(N));
    if (tid == 0) {
        for (int i = 0; i < NS; ++i) mbar_init(&bar[i], 1);
        mbar_init_fence();
    }
    // voxel records of the first NS - 1 stages
    for (int s = 0; s < NS - 1 && s < n_stages; ++s)
        if (tid < KSTAGE) s_vox[s][tid] = make_vox(v_begin + (long long)s * KSTAGE + tid, v_end, S);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t sbase = smem_u32(smem);
    constexpr uint32_t IDESC = idesc_bf16(TILE_M, N, 1, 1);

    // this thread's A row group (8 channels of one tap) is fixed
    const int g = (tid >> 3) & (TILE_M / 8 - 1);
    const int r = r0 + g * 8;
    const bool row_in = r < rows;
    const int tap = row_in ? r / cin : 0, ci = row_in ? r - tap * cin : 0;
    const int req = tap_req(tap);
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    const bool from_a = ci < S.ca;
    const long long a_off = (long long)((dz * S.H + dy) * S.W + dx);   // neighbour offset in voxels
    const int klo = tid & 7, khi0 = tid >> 7;

    auto issue = [&](int s) {
        const int buf = s % NS;
        const uint32_t sa = sbase + (uint32_t)buf * STAGE, sb = sa + A_BYTES;
        // A (MN-major): voxel k, row group g at (k / 8) * (TILE_M * 16) + g * 128 + (k % 8) * 16
#pragma unroll
        for (int j = 0; j < TILE_M / 8 * KSTAGE / THREADS; ++j) {
            const int khi = khi0 + 2 * j, k = khi * 8 + klo;
            const VoxRec vr = s_vox[buf][k];
            uint32_t bytes = 0;
            const void* src = S.a;
            if (row_in && vr.v >= 0 && (vr.flags & req) == req) {
                bytes = 16;
                if (from_a) {
                    src = S.a + ((long long)vr.v + a_off) * S.ca + ci;
                } else {
                    const int cz = (((vr.par >> 2) & 1) + dz) >> 1, cy = (((vr.par >> 1) & 1) + dy) >> 1,
                              cx = ((vr.par & 1) + dx) >> 1;
                    src = S.b + (size_t)(vr.cv + (cz * (S.H >> 1) + cy) * (S.W >> 1) + cx) * S.cb + (ci - S.ca);
                }
            }
            cp_async16(sa + khi * (TILE_M * 16) + g * 128 + klo * 16, src, bytes);
        }
        // B (MN-major): voxel k, output-channel group gg at (k / 8) * (N * 16) + gg * 128 + (k % 8) * 16
        for (int i = tid; i < N / 8 * KSTAGE; i += THREADS) {
            const int kl = i & 7, gg = (i >> 3) % (N / 8), kh = i / N;
            const int v = s_vox[buf][kh * 8 + kl].v;
            cp_async16(sb + kh * (N * 16) + gg * 128 + kl * 16,
                       v >= 0 ? (const void*)(P.dz + (size_t)v * N + gg * 8) : (const void*)P.dz, v >= 0 ? 16u : 0u);
        }
    };

    bool ok = true;
    int issued = 0;
    for (int s = 0; s < NS - 1; ++s) {
        if (s < n_stages) issue(s);
        cp_async_commit();
    }
    for (int it = 0; it < n_stages; ++it) {
        cp_async_wait<NS - 2>();
        fence_proxy_async();
        // records of stage it + NS - 1: their buffer was last read when stage
        // it - 1 was issued, before the previous barrier
        const int nxt = it + NS - 1;
        if (nxt < n_stages && tid < KSTAGE)
            s_vox[nxt % NS][tid] = make_vox(v_begin + (long long)nxt * KSTAGE + tid, v_end, S);
        if (!__syncthreads_and(ok)) { ok = false; break; }
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = sbase + (uint32_t)(it % NS) * STAGE, b0 = a0 + A_BYTES;
#pragma unroll
            for (int k = 0; k < KSTAGE / 16; ++k) {
                uint64_t ad = smem_desc(a0 + k * 2 * (TILE_M * 16), TILE_M * 16, 128);
                uint64_t bd = smem_desc(b0 + k * 2 * (N * 16), N * 16, 128);
                mma_bf16(tmem, ad, bd, IDESC, (it > 0 || k > 0) ? 1u : 0u);
            }
            mma_commit(&bar[it % NS]);
        }
        issued = it + 1;
        if (nxt < n_stages) {
            if (it >= 1) ok = mbar_wait(&bar[(it - 1) % NS], ((it - 1) / NS) & 1);
            if (ok) issue(nxt);
        }
        cp_async_commit();
    }
    cp_async_wait<0>();
    if (issued > 0 && !mbar_wait(&bar[(issued - 1) % NS], ((issued - 1) / NS) & 1)) ok = false;
    ok = __syncthreads_and(ok && issued == n_stages);
    tc_fence_after();

    if (ok && n_stages > 0) {
        const int q = warp & 3, half = warp >> 2;
        const int rr = r0 + q * 32 + lane;
        const int tp = rr / cin, cc = rr - tp * cin;
        for (int c0 = half * 8; c0 < N; c0 += 16) {
            float f[8];
            tmem_ld8(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, f);
            if (rr < rows) {
#pragma unroll
                for (int j = 0; j < 8; ++j) atomicAdd(P.dw + ((size_t)tp * N + c0 + j) * cin + cc, f[j]);
            }
        }
    } else if (!ok && tid == 0) {
        atomicOr(&g_status, 1u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, tmem_cols(N));
}

// ---------------------------------------------------------------------------
// weight gradient from tensor-memory-accelerator tile loads
// ---------------------------------------------------------------------------

// The GEMM of wgrad_kernel -- M = 128 (tap, ci) rows, N = output channels,
// K = voxels -- for inputs that are not concatenated, with both operands
// copied by the tensor memory accelerator instead of gathered by threads.
// A K stage is a block of bx x by = 64 voxels at one z (bx a power of two
// that divides W).  A box {c channels, bx, by, 1, 1} of the input, c =
// min(cin, 64), at the stage's coordinates shifted by one tap holds the
// A operand of c rows (tap, ci0 .. ci0 + c - 1) of the M tile: 64 voxel
// rows of 2c bytes, written with the 32-, 64- or 128-byte swizzle that
// matches its row length, which is the MN-major swizzled layout of the MMA
// (the M tile's 128 / c boxes are its atom columns, 128 c bytes apart; K
// groups of 8 rows are 16 c bytes apart).  The copy engine handles a box
// row per cycle or so, so rows of whole voxels (32 bytes and more) move
// more bytes per row than 16-byte channel groups would.  Coordinates
// outside the volume read zeros, the convolution's zero padding.  The
// output-gradient operand is the same kind of box of dz at the unshifted
// coordinates (min(N, 64) channels), so K runs over the same voxels in the
// same order in both.  Warp 0 issues the copies (lanes 0 .. 7: A boxes;
// lanes 16, 17: dz boxes) once lane 0 has set the stage's expected bytes;
// one thread of warp 1 issues the MMAs and commits the stage's "empty"
// barrier; every warp then reads the accumulator and adds it into dw.
struct WgradT {
    float* dw;                   // [27][N][ld], accumulated at columns c_off .. c_off + cin - 1
    int ld, c_off;               // columns of dw (all input channels of the layer), first column here
    int cin, rows;               // input channels of this operand, 27 x cin
    int a_ch;                    // channels of an A box: min(cin, 64)
    int D, ny_blk, nx_blk;       // depth, y blocks (of by), x blocks (of bx)
    int bx, by;                  // a stage's voxels along x and y (bx x by = KSTAGE)
    long long stages;            // volumes x D x ny_blk x nx_blk
};

__host__ __device__ constexpr int wgrad_tma_stages(int n) { return n <= 16 ? 6 : (n <= 32 ? 5 : (n <= 64 ? 4 : 3)); }
// descriptor layout type of rows of `bytes` (32, 64 or 128)
__host__ __device__ constexpr uint32_t swizzle_layout(int bytes) { return bytes == 32 ? 6u : (bytes == 64 ? 4u : 2u); }

template <int N>
__global__ void __launch_bounds__(THREADS) wgrad_tma_kernel(const __grid_constant__ CUtensorMap xmap,
                                                            const __grid_constant__ CUtensorMap zmap,
                                                            const WgradT P) {
    constexpr int NS = wgrad_tma_stages(N);
    constexpr int B_CH = N < 64 ? N : 64;                      // channels of a dz box
    constexpr uint32_t A_BYTES = TILE_M * KSTAGE * 2, STAGE = wgrad_stage_bytes(N);
    static_assert(STAGE % 1024 == 0, "stages keep the 1 KB alignment of the swizzle patterns");
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ uint64_t full[NS], empty[NS], done;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int r0 = blockIdx.x * TILE_M;
    const long long s_begin = P.stages * blockIdx.y / gridDim.y;
    const int n_st = (int)(P.stages * (blockIdx.y + 1) / gridDim.y - s_begin);
    volatile int* fail = &s_fail;

    if (warp == 0) tmem_alloc(&s_tmem, tmem_cols(N));
    if (tid == 0) {
        for (int i = 0; i < NS; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(&done, 1);
        s_fail = 0;
        mbar_init_fence();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t sbase = (smem_u32(smem) + 1023u) & ~1023u;     // the launch adds 1 KB of slack

    if (warp == 0) {
        // ---- copies: this lane's box, fixed for the CTA ----
        int c0 = 0, ox = 0, oy = 0, oz = 0;
        uint32_t dst = 0, box = 0;                                // box bytes, 0: no box
        const CUtensorMap* map = &xmap;
        if (lane < TILE_M / P.a_ch) {
            const int r = r0 + lane * P.a_ch;
            if (r < P.rows) {
                const int tap = r / P.cin;
                c0 = r - tap * P.cin;
                oz = tap / 9 - 1;
                oy = (tap / 3) % 3 - 1;
                ox = tap % 3 - 1;
                box = (uint32_t)(KSTAGE * 2 * P.a_ch);
                dst = (uint32_t)lane * box;
            }
        } else if (lane >= 16 && lane < 16 + N / B_CH) {
            c0 = (lane - 16) * B_CH;
            box = (uint32_t)(KSTAGE * 2 * B_CH);
            dst = A_BYTES + (uint32_t)(lane - 16) * box;
            map = &zmap;
        }
        const uint32_t bytes = __reduce_add_sync(0xffffffffu, box);
        int issued = 0;
        for (int s = 0; s < n_st; ++s) {
            const int slot = s % NS;
            int ok = 1;
            // the slot's previous stage has been read by its MMAs
            if (lane == 0 && s >= NS) ok = mbar_wait_or_fail(&empty[slot], (uint32_t)((s / NS) - 1) & 1u, fail);
            if (!__shfl_sync(0xffffffffu, ok, 0)) break;
            long long q = s_begin + s;
            const int xb = (int)(q % P.nx_blk);
            q /= P.nx_blk;
            const int yb = (int)(q % P.ny_blk);
            q /= P.ny_blk;
            const int z = (int)(q % P.D), n = (int)(q / P.D);
            if (lane == 0) mbar_arrive_expect_tx(&full[slot], bytes);
            __syncwarp();
            if (box)
                tma_load_5d(sbase + (uint32_t)slot * STAGE + dst, map, &full[slot], c0, xb * P.bx + ox,
                            yb * P.by + oy, z + oz, n);
            issued = s + 1;
        }
        // after a failure, the copies still in flight land before the CTA ends
        if (lane == 0 && *fail)
            for (int s = max(0, issued - NS); s < issued; ++s) mbar_wait(&full[s % NS], (uint32_t)(s / NS) & 1u);
    } else if (warp == 1 && lane == 0) {
        // ---- MMAs: four of K = 16 voxels per stage ----
        constexpr uint32_t IDESC = idesc_bf16(TILE_M, N, 1, 1);
        const uint32_t ar = 2u * (uint32_t)P.a_ch, al = swizzle_layout((int)ar);      // A row bytes, layout
        constexpr uint32_t BR = 2u * B_CH, BL = swizzle_layout(2 * B_CH);
        for (int s = 0; s < n_st; ++s) {
            const int slot = s % NS;
            if (!mbar_wait_or_fail(&full[slot], (uint32_t)(s / NS) & 1u, fail)) break;
            tc_fence_after();
            const uint32_t a0 = sbase + (uint32_t)slot * STAGE, b0 = a0 + A_BYTES;
#pragma unroll
            for (int k = 0; k < KSTAGE / 16; ++k)
                mma_bf16(tmem, smem_desc_sw(a0 + k * 16 * ar, KSTAGE * ar, 8 * ar, al),
                         smem_desc_sw(b0 + k * 16 * BR, KSTAGE * BR, 8 * BR, BL), IDESC, (s > 0 || k > 0) ? 1u : 0u);
            mma_commit(&empty[slot]);
        }
        mma_commit(&done);          // arrives once every MMA issued above has finished
    }
    // ---- epilogue: the accumulator into dw ----
    if (lane == 0) mbar_wait_or_fail(&done, 0u, fail);
    __syncthreads();
    tc_fence_after();
    const bool good = !*fail && n_st > 0;
    if (good) {
        const int q = warp & 3, half = warp >> 2;
        const int rr = r0 + q * 32 + lane;
        const int tp = rr / P.cin, cc = rr - tp * P.cin;
        for (int c0 = half * 8; c0 < N; c0 += 16) {
            float f[8];
            tmem_ld8(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, f);
            if (rr < P.rows) {
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    atomicAdd(P.dw + ((size_t)tp * N + c0 + j) * P.ld + P.c_off + cc, f[j]);
            }
        }
    } else if (*fail && tid == 0) {
        atomicOr(&g_status, 1u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, tmem_cols(N));
}

// Nearest 2x upsampling, channels-last: out[n][z][y][x] = b[n][z/2][y/2][x/2]
// (the second input of a concatenated layer, spelled out for the tile loads).
__global__ void upsample_kernel(const uint4* __restrict__ b, uint4* __restrict__ out, int batch, int d, int h,
                                int w, int c8) {
    const long long total = (long long)batch * d * h * w * c8;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % c8);
        long long v = i / c8;
        const int x = (int)(v % w);
        v /= w;
        const int y = (int)(v % h);
        v /= h;
        const int z = (int)(v % d);
        const long long n = v / d;
        const long long cv = ((n * (d >> 1) + (z >> 1)) * (h >> 1) + (y >> 1)) * (w >> 1) + (x >> 1);
        out[i] = __ldg(b + cv * c8 + c);
    }
}

// ---------------------------------------------------------------------------
// memory-bound helpers (CUDA cores)
// ---------------------------------------------------------------------------

// db[c] += sum_v dz[v][c]
__global__ void bias_grad_kernel(const __nv_bfloat16* __restrict__ dz, long long n_vox, int c,
                                 float* __restrict__ db) {
    extern __shared__ float s_acc[];
    for (int i = threadIdx.x; i < c; i += blockDim.x) s_acc[i] = 0.0f;
    __syncthreads();
    const long long total = n_vox * c;
    float acc = 0.0f;
    int cur = -1;
    // blockDim.x is a multiple of c, so every thread sums a single channel
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        cur = (int)(i % c);
        acc += __bfloat162float(dz[i]);
    }
    if (cur >= 0) atomicAdd(&s_acc[cur], acc);
    __syncthreads();
    for (int i = threadIdx.x; i < c; i += blockDim.x) atomicAdd(db + i, s_acc[i]);
}

// y[n, z, y, x, c] = mean of the 2x2x2 children (D, H, W of x even)
__global__ void avgpool_kernel(const __nv_bfloat16* __restrict__ x, int B, int D, int H, int W, int c,
                               __nv_bfloat16* __restrict__ y) {
    const int D2 = D >> 1, H2 = H >> 1, W2 = W >> 1;
    const long long total = (long long)B * D2 * H2 * W2 * (c >> 3);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c8 = (int)(i % (c >> 3));
        long long v = i / (c >> 3);
        const int xx = (int)(v % W2);
        long long t = v / W2;
        const int yy = (int)(t % H2);
        t /= H2;
        const int zz = (int)(t % D2);
        const int n = (int)(t / D2);
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 8; ++k) {
            size_t src = ((((size_t)n * D + 2 * zz + (k >> 2)) * H + 2 * yy + ((k >> 1) & 1)) * W + 2 * xx + (k & 1)) * c +
                         c8 * 8;
            float f[8];
            unpack_bf16x8(__ldg(reinterpret_cast<const uint4*>(x + src)), f);
#pragma unroll
            for (int j = 0; j < 8; ++j) s[j] += f[j];
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) s[j] *= 0.125f;
        *reinterpret_cast<uint4*>(y + (size_t)v * c + c8 * 8) = pack_bf16x8(s);
    }
}

// dz_x[v][c] += (x_act[v][c] > 0) * gy[parent(v)][c] / 8   (x at full resolution)
__global__ void pool_backward_kernel(const __nv_bfloat16* __restrict__ gy, const __nv_bfloat16* __restrict__ x_act,
                                     int B, int D, int H, int W, int c, __nv_bfloat16* __restrict__ dz_x) {
    const long long total = (long long)B * D * H * W * (c >> 3);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c8 = (int)(i % (c >> 3));
        long long v = i / (c >> 3);
        const int xx = (int)(v % W);
        long long t = v / W;
        const int yy = (int)(t % H);
        t /= H;
        const int zz = (int)(t % D);
        const int n = (int)(t / D);
        size_t p = ((((size_t)n * (D >> 1) + (zz >> 1)) * (H >> 1) + (yy >> 1)) * (W >> 1) + (xx >> 1)) * c + c8 * 8;
        size_t o = (size_t)v * c + c8 * 8;
        float g[8], a[8], d[8];
        unpack_bf16x8(__ldg(reinterpret_cast<const uint4*>(gy + p)), g);
        unpack_bf16x8(__ldg(reinterpret_cast<const uint4*>(x_act + o)), a);
        unpack_bf16x8(*reinterpret_cast<const uint4*>(dz_x + o), d);
#pragma unroll
        for (int j = 0; j < 8; ++j) d[j] += a[j] > 0.0f ? 0.125f * g[j] : 0.0f;
        *reinterpret_cast<uint4*>(dz_x + o) = pack_bf16x8(d);
    }
}

// dz_c[vc][c] = (coarse_act[vc][c] > 0) * sum over the 8 children of g_full
// (g_full at full resolution D, H, W)
__global__ void up_reduce_kernel(const __nv_bfloat16* __restrict__ g_full, const __nv_bfloat16* __restrict__ coarse,
                                 int B, int D, int H, int W, int c, __nv_bfloat16* __restrict__ dz_c) {
    const int D2 = D >> 1, H2 = H >> 1, W2 = W >> 1;
    const long long total = (long long)B * D2 * H2 * W2 * (c >> 3);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c8 = (int)(i % (c >> 3));
        long long v = i / (c >> 3);
        const int xx = (int)(v % W2);
        long long t = v / W2;
        const int yy = (int)(t % H2);
        t /= H2;
        const int zz = (int)(t % D2);
        const int n = (int)(t / D2);
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 8; ++k) {
            size_t src = ((((size_t)n * D + 2 * zz + (k >> 2)) * H + 2 * yy + ((k >> 1) & 1)) * W + 2 * xx + (k & 1)) * c +
                         c8 * 8;
            float f[8];
            unpack_bf16x8(__ldg(reinterpret_cast<const uint4*>(g_full + src)), f);
#pragma unroll
            for (int j = 0; j < 8; ++j) s[j] += f[j];
        }
        float a[8];
        size_t o = (size_t)v * c + c8 * 8;
        unpack_bf16x8(__ldg(reinterpret_cast<const uint4*>(coarse + o)), a);
#pragma unroll
        for (int j = 0; j < 8; ++j) s[j] = a[j] > 0.0f ? s[j] : 0.0f;
        *reinterpret_cast<uint4*>(dz_c + o) = pack_bf16x8(s);
    }
}

// Head (1x1x1 conv, 16 -> 1, residual on the input log-kerma) with the
// weighted squared-error loss and, when dz is given, its backward:
//   out = xlog + head[0:16] . d0 + head[16]
//   loss = sum_v wgt (out - tgt)^2 * inv_wsum
//   dz_d0 = (d0 > 0) * dout * head[0:16],  dout = 2 wgt (out - tgt) inv_wsum
// dhead[0..15] += dL/dweights, dhead[16] += dL/dbias, loss[0] += loss.
__global__ void head_kernel(const __nv_bfloat16* __restrict__ d0, const float* __restrict__ xlog,
                            const float* __restrict__ tgt, const float* __restrict__ wgt,
                            const float* __restrict__ head, float inv_wsum, long long n_vox, float* __restrict__ out,
                            __nv_bfloat16* __restrict__ dz, float* __restrict__ dhead, float* __restrict__ loss) {
    __shared__ float s_acc[18];
    if (threadIdx.x < 18) s_acc[threadIdx.x] = 0.0f;
    __syncthreads();
    float w[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) w[j] = __ldg(head + j);
    const float hb = __ldg(head + 16);
    float g[18];
#pragma unroll
    for (int j = 0; j < 18; ++j) g[j] = 0.0f;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n_vox;
         v += (long long)gridDim.x * blockDim.x) {
        float a[16];
        unpack_bf16x8(__ldg(reinterpret_cast<const uint4*>(d0 + (size_t)v * 16)), a);
        unpack_bf16x8(__ldg(reinterpret_cast<const uint4*>(d0 + (size_t)v * 16 + 8)), a + 8);
        float o = xlog[v] + hb;
#pragma unroll
        for (int j = 0; j < 16; ++j) o += w[j] * a[j];
        if (out) out[v] = o;
        if (tgt) {
            const float wv = wgt ? wgt[v] : 1.0f;
            const float e = o - tgt[v];
            g[17] += wv * e * e * inv_wsum;
            const float dout = 2.0f * wv * e * inv_wsum;
            if (dz) {
                float d[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    d[j] = a[j] > 0.0f ? dout * w[j] : 0.0f;
                    g[j] += dout * a[j];
                }
                *reinterpret_cast<uint4*>(dz + (size_t)v * 16) = pack_bf16x8(d);
                *reinterpret_cast<uint4*>(dz + (size_t)v * 16 + 8) = pack_bf16x8(d + 8);
                g[16] += dout;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 18; ++j) {
        float t = g[j];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if ((threadIdx.x & 31) == 0 && t != 0.0f) atomicAdd(&s_acc[j], t);
    }
    __syncthreads();
    if (threadIdx.x < 17 && dhead && s_acc[threadIdx.x] != 0.0f) atomicAdd(dhead + threadIdx.x, s_acc[threadIdx.x]);
    if (threadIdx.x == 17 && loss && s_acc[17] != 0.0f) atomicAdd(loss, s_acc[17]);
}

// Network input: 16 channels per voxel -- normalised log kerma, density,
// material one-hot (n_mat <= 13), zeros, and in channel 15 the input map's
// relative standard error when given.
__global__ void input_kernel(const float* __restrict__ xlog, const float* __restrict__ density,
                             const uint8_t* __restrict__ mat, int n_mat, const float* __restrict__ unc, long long n_vox,
                             __nv_bfloat16* __restrict__ x) {
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n_vox;
         v += (long long)gridDim.x * blockDim.x) {
        float f[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) f[j] = 0.0f;
        f[0] = xlog[v];
        f[1] = density[v];
        const int m = mat[v];
        if (m < n_mat && m < 13) f[2 + m] = 1.0f;
        if (unc) f[15] = unc[v];
        *reinterpret_cast<uint4*>(x + (size_t)v * 16) = pack_bf16x8(f);
        *reinterpret_cast<uint4*>(x + (size_t)v * 16 + 8) = pack_bf16x8(f + 8);
    }
}

// Adam with decoupled weight decay on a flat FP32 parameter vector.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                            float c2, float wd, const double* __restrict__ clip) {
    const float scale = clip ? (float)clip[2] : 1.0f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i] * scale;
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * ((mi * c1) / (sqrtf(vi * c2) + eps) + wd * p[i]);
    }
}

// Sum of squares of g[0, n) added to *out (block partials in FP64).
__global__ void sumsq_kernel(const float* __restrict__ g, long long n, double* __restrict__ out) {
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double x = g[i];
        s += x * x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = (threadIdx.x < (blockDim.x >> 5)) ? part[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) atomicAdd(out, s);
    }
}

// Adaptive global-norm clipping, state [sumsq, ema, scale]: the gradient's
// norm is capped at ratio x the running mean of the capped norms (the first
// step sets that mean), so that one outlying minibatch cannot inflate
// Adam's second moments or throw the weights far.
__global__ void clip_scale_kernel(double* state, float ratio) {
    const double norm = sqrt(state[0]);
    double ema = state[1];
    if (!(ema > 0.0)) ema = norm;
    const double cap = ratio * ema;
    const double kept = norm > cap ? cap : norm;
    state[2] = norm > 0.0 ? kept / norm : 1.0;
    state[1] = 0.95 * ema + 0.05 * kept;
}

// BF16 weights of one layer from its FP32 master copy w32[27][cout][cin],
// packed in tile order (packed_elems): wp for the forward convolution
// (n = cout, c = cin, W(tap, r, ch) = w32[tap][r][ch]) and wtp for the
// backward-data convolution (n = cin, c = cout, W(tap, r, ch) =
// w32[26 - tap][ch][r]: flipped taps, transposed channels).
__global__ void pack_weights_kernel(const float* __restrict__ w32, int cout, int cin, __nv_bfloat16* __restrict__ wp,
                                    __nv_bfloat16* __restrict__ wtp) {
    const long long nf = packed_elems(cout, cin), nb = wtp ? packed_elems(cin, cout) : 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nf + nb;
         i += (long long)gridDim.x * blockDim.x) {
        const bool fwd = i < nf;
        const long long j = fwd ? i : i - nf;
        const int n = fwd ? cout : cin, c = fwd ? cin : cout;
        const int e = (int)(j & 7);
        long long t = j >> 3;
        const int r = (int)(t % n);
        t /= n;
        const int c8 = (int)(t & 7);
        const long long st = t >> 3;
        const long long k = st * KS + c8 * 8 + e;
        const int tap = (int)(k / c), ch = (int)(k - (long long)tap * c);
        float val = 0.0f;
        if (tap < 27) val = fwd ? w32[((size_t)tap * cout + r) * cin + ch] : w32[((size_t)(26 - tap) * cout + ch) * cin + r];
        (fwd ? wp : wtp)[j] = __float2bfloat16_rn(val);
    }
}

// Plain tensor-core GEMM D[M][N] = A[M][K] . B[N][K]^T for the unit tests of
// the descriptors (A, B K-major BF16; D FP32; M a multiple of 128, N of 16
// up to 256, K of 64).
__global__ void __launch_bounds__(THREADS) gemm_test_kernel(const __nv_bfloat16* A, const __nv_bfloat16* Bm,
                                                            float* Dm, int M, int N, int K, int a_mn, int b_mn) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TILE_M;
    if (warp == 0) tmem_alloc(&s_tmem, 256);
    if (tid == 0) {
        mbar_init(&bar, 1);
        mbar_init_fence();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    uint8_t* sA = smem;
    uint8_t* sB = smem + TILE_M * 64 * 2;
    bool ok = true;
    const uint32_t idesc = idesc_bf16(TILE_M, N, a_mn, b_mn);
    for (int k0 = 0; k0 < K && ok; k0 += 64) {
        // K-major: row r, chunk c8 at c8 * (rows * 16) + (r / 8) * 128 + (r % 8) * 16
        // MN-major: k, group g at (k / 8) * (rows * 16) + g * 128 + (k % 8) * 16 (A given as [K][M])
        for (int i = tid; i < TILE_M * 8; i += THREADS) {
            if (!a_mn) {
                const int r = i & (TILE_M - 1), c8 = i >> 7;
                *reinterpret_cast<uint4*>(sA + c8 * (TILE_M * 16) + (r >> 3) * 128 + (r & 7) * 16) =
                    *reinterpret_cast<const uint4*>(A + (size_t)(m0 + r) * K + k0 + c8 * 8);
            } else {
                const int klo = i & 7, g = (i >> 3) & 15, khi = i >> 7;
                *reinterpret_cast<uint4*>(sA + khi * (TILE_M * 16) + g * 128 + klo * 16) =
                    *reinterpret_cast<const uint4*>(A + (size_t)(k0 + khi * 8 + klo) * M + m0 + g * 8);
            }
        }
        for (int i = tid; i < N * 8; i += THREADS) {
            if (!b_mn) {
                const int r = i % N, c8 = i / N;
                *reinterpret_cast<uint4*>(sB + c8 * (N * 16) + (r >> 3) * 128 + (r & 7) * 16) =
                    *reinterpret_cast<const uint4*>(Bm + (size_t)r * K + k0 + c8 * 8);
            } else {
                const int klo = i & 7, g = (i >> 3) % (N / 8), khi = i / N;
                *reinterpret_cast<uint4*>(sB + khi * (N * 16) + g * 128 + klo * 16) =
                    *reinterpret_cast<const uint4*>(Bm + (size_t)(k0 + khi * 8 + klo) * N + g * 8);
            }
        }
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            for (int k = 0; k < 4; ++k) {
                uint64_t ad = smem_desc(smem_u32(sA) + k * 2 * (TILE_M * 16), TILE_M * 16, 128);
                uint64_t bd = smem_desc(smem_u32(sB) + k * 2 * (N * 16), N * 16, 128);
                mma_bf16(tmem, ad, bd, idesc, (k0 > 0 || k > 0) ? 1u : 0u);
            }
            mma_commit(&bar);
        }
        ok = mbar_wait(&bar, (k0 / 64) & 1);
        ok = __syncthreads_and(ok);
        tc_fence_after();
    }
    if (ok) {
        const int q = warp & 3, half = warp >> 2;
        for (int c0 = half * 8; c0 < N; c0 += 16) {
            float f[8];
            tmem_ld8(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, f);
            for (int j = 0; j < 8; ++j) Dm[(size_t)(m0 + q * 32 + lane) * N + c0 + j] = f[j];
        }
    } else if (tid == 0) {
        atomicOr(&g_status, 1u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 256);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

int g_sm_count = 0;

int sm_count() {
    if (g_sm_count == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return 148;
        cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        if (g_sm_count <= 0) g_sm_count = 148;
    }
    return g_sm_count;
}

int grid_for(long long work, int threads) {
    long long b = (work + threads - 1) / threads;
    long long cap = (long long)sm_count() * 16;
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// Shared memory per CTA: the pipeline stages, raised where needed so that
// the CTAs resident on one SM never ask for more than its 512 tensor-memory
// columns together (an allocation beyond that would wait for another CTA).
template <typename K>
int tc_launch_smem(K kernel, size_t stages_bytes, uint32_t cols, size_t& smem) {
    smem = stages_bytes;
    const int max_ctas = (int)(512u / cols);
    int dev = 0;
    CU_CHECK(cudaGetDevice(&dev));
    int per_sm = 0;
    CU_CHECK(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    const size_t floor_smem = (size_t)per_sm / (size_t)(max_ctas + 1) + 1024;
    if (smem < floor_smem) smem = floor_smem;
    if (smem > 200 * 1024) return set_error(CCU_E_INVALID, "stages too large for shared memory");
    CU_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CU_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared));
    int occ = 0;
    CU_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, THREADS, smem));
    if (occ * (int)cols > 512) return set_error(CCU_E_INVALID, "tensor-memory budget per SM exceeded");
    if (occ < 1) return set_error(CCU_E_INVALID, "kernel does not fit on an SM");
    return CCU_OK;
}

template <int N>
int launch_conv(const ConvP& P, cudaStream_t st) {
    size_t smem = 0;
    int rc = tc_launch_smem(conv_kernel<N>, (size_t)CONV_STAGES * conv_stage_bytes(N), tmem_cols(N), smem);
    if (rc != CCU_OK) return rc;
    const long long blocks = (P.n_vox + TILE_M - 1) / TILE_M;
    conv_kernel<N><<<(unsigned)blocks, THREADS, smem, st>>>(P);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

// 0: the plane-stationary kernel where it applies, else the streaming halo
// kernel where it applies, else the gathering kernel; 1: always the
// gathering kernel; 2: the one-tile halo kernel where it applies; 3: the
// warp-role streaming kernel where the streaming kernel applies; 4: path 0
// without the plane-stationary kernel
int g_conv_path = 0;

bool halo_applies(const ConvP& P, int n_out) {
    const int cin = P.src.ca + P.src.cb;
    return g_conv_path == 2 && P.src.H % 16 == 0 && P.src.W % 8 == 0 && cin <= 48 && n_out <= 48 &&
           halo_smem_bytes(n_out, cin) <= 160 * 1024;
}

bool stream_applies(const ConvP& P, int n_out) {
    const int cin = P.src.ca + P.src.cb;
    return (g_conv_path == 0 || g_conv_path == 3 || g_conv_path == 4) && cin <= 48 && n_out <= 48 &&
           stream_smem_bytes(n_out, cin) <= 200 * 1024;
}

// Channel passes of the plane-stationary kernel for cin input channels: the
// fewest passes of equal 16-channel-aligned groups whose weights and a
// ring of 3 planes fit 200 KB of shared memory (0: does not apply).
// Output slices of the plane-stationary kernel: one of 16 or 32 channels,
// two of 32 for 64 (0: does not apply).
int ps_slice(int n_out) {
    if (g_conv_path != 0) return 0;
    return n_out == 16 ? 16 : (n_out == 32 || n_out == 64) ? 32 : 0;
}

int ps_passes(int n_out, int cin) {
    const int no = ps_slice(n_out);
    if (!no || cin % 16) return 0;
    const int c16 = cin / 16;
    for (int passes = 1; passes <= c16; ++passes) {
        const int c8p = 2 * ((c16 + passes - 1) / passes);
        if (ps_smem_bytes(no, c8p, 3) <= 200 * 1024) return passes;
    }
    return 0;
}

// Resident CTAs per SM of a kernel launched with THREADS threads and this
// dynamic shared memory: shared memory (1 KB of it reserved per CTA), the
// registers of its threads, the 512 tensor-memory columns and the 2048
// threads of an SM.
template <typename Kern>
int resident_ctas(Kern kernel, size_t smem, uint32_t cols, int& resident) {
    int dev = 0, per_sm = 0;
    CU_CHECK(cudaGetDevice(&dev));
    CU_CHECK(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    cudaFuncAttributes fa;
    CU_CHECK(cudaFuncGetAttributes(&fa, kernel));
    const int regs = ((std::max(fa.numRegs, 1) + 7) / 8) * 8;      // allocated per thread in steps of 8
    resident = std::max(1, std::min({(int)((size_t)per_sm / (smem + 1024)), 65536 / (regs * THREADS),
                                     (int)(512u / cols), 2048 / THREADS}));
    return CCU_OK;
}

// ring depth of the warp-role kernel (0: chosen per layer)
int g_conv_ring = 0;
// issue group of the plane-stationary kernel (0: chosen per layer)
int g_conv_group = 0;

template <int N>
int launch_conv_stream(const ConvP& P, cudaStream_t st) {
    const int cin = P.src.ca + P.src.cb;
    int dev = 0, sms = 0;
    CU_CHECK(cudaGetDevice(&dev));
    CU_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    size_t smem = 0;
    int rc = CCU_OK, resident = 1;
    if (g_conv_path == 3) {
        // deepest useful ring: most planes in flight per SM (resident CTAs x
        // the ring - 3 planes each copies ahead of its MMAs)
        const long long planes = (long long)P.src.B * ((P.src.H + 15) / 16) * ((P.src.W + 7) / 8) * P.src.D;
        int ring = g_conv_ring;
        if (ring == 0) {
            int per_sm = 0, best = -1;
            CU_CHECK(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
            // tc_launch_smem's floor: no more CTAs per SM than the tensor memory holds
            const size_t floor_smem = (size_t)per_sm / (512u / stream_tmem_cols(N) + 1) + 1024;
            for (int r = 4; r <= WS_RING_MAX && ws_smem_bytes(N, cin, r) <= 200 * 1024; ++r) {
                int res = 1;
                rc = resident_ctas(conv_ws_kernel<N>, std::max<size_t>(ws_smem_bytes(N, cin, r), floor_smem),
                                   stream_tmem_cols(N), res);
                if (rc != CCU_OK) return rc;
                if (res * (r - 3) > best) best = res * (r - 3), ring = r;
            }
        }
        if (ws_smem_bytes(N, cin, ring) > 200 * 1024) return set_error(CCU_E_INVALID, "ring too deep for this layer");
        rc = tc_launch_smem(conv_ws_kernel<N>, ws_smem_bytes(N, cin, ring), stream_tmem_cols(N), smem);
        if (rc != CCU_OK) return rc;
        if ((rc = resident_ctas(conv_ws_kernel<N>, smem, stream_tmem_cols(N), resident)) != CCU_OK) return rc;
        const long long grid = std::min<long long>(planes, (long long)sms * resident);
        conv_ws_kernel<N><<<(unsigned)grid, THREADS, smem, st>>>(P, ring);
        CU_CHECK(cudaGetLastError());
        return CCU_OK;
    }
    rc = tc_launch_smem(conv_stream_kernel<N>, stream_smem_bytes(N, cin), stream_tmem_cols(N), smem);
    if (rc != CCU_OK) return rc;
    const long long items = (long long)P.src.B * ((P.src.H + 15) / 16) * ((P.src.W + 7) / 8) *
                            ((P.src.D + ZSEG - 1) / ZSEG);
    if (items >= (1LL << 31)) return set_error(CCU_E_INVALID, "volume too large");
    if ((rc = resident_ctas(conv_stream_kernel<N>, smem, stream_tmem_cols(N), resident)) != CCU_OK) return rc;
    const long long grid = std::min<long long>(items, (long long)sms * resident);
    conv_stream_kernel<N><<<(unsigned)grid, THREADS, smem, st>>>(P, (int)items);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

// FP32 partial sums of multi-pass plane-stationary convolutions: one
// buffer per device, grown on demand (the stream is drained before an
// older, smaller buffer is freed) and kept for the process.
struct DevBuffers {
    std::mutex mu;
    void* p[64] = {};
    size_t bytes[64] = {};
};
DevBuffers g_ws;          // FP32 partial sums of channel passes
DevBuffers g_up_ws;       // the upsampled input of a weight gradient

int grow_buffer(DevBuffers& b, size_t bytes, cudaStream_t st, void*& out) {
    int dev = 0;
    CU_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(CCU_E_INVALID, "device index out of range");
    std::lock_guard<std::mutex> lk(b.mu);
    if (b.bytes[dev] < bytes) {
        if (b.p[dev]) {
            CU_CHECK(cudaStreamSynchronize(st));
            CU_CHECK(cudaFree(b.p[dev]));
            b.p[dev] = nullptr;
            b.bytes[dev] = 0;
        }
        CU_CHECK(cudaMalloc(&b.p[dev], bytes));
        b.bytes[dev] = bytes;
    }
    out = b.p[dev];
    return CCU_OK;
}

int ps_workspace(size_t bytes, cudaStream_t st, float*& ws) {
    void* p = nullptr;
    const int rc = grow_buffer(g_ws, bytes, st, p);
    ws = (float*)p;
    return rc;
}

template <int NO, int G>
int launch_conv_ps_g(const ConvP& P, int n_out, int passes, cudaStream_t st) {
    const int c8n = (P.src.ca + P.src.cb) / 8;
    const int c8p_max = 2 * ((c8n / 2 + passes - 1) / passes);
    int dev = 0, sms = 0;
    CU_CHECK(cudaGetDevice(&dev));
    CU_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long long planes = (long long)P.src.B * ((P.src.H + 15) / 16) * ((P.src.W + 7) / 8) * P.src.D;
    float* ws = nullptr;
    if (passes > 1) {
        const int rc = ps_workspace((size_t)P.n_vox * NO * sizeof(float), st, ws);
        if (rc != CCU_OK) return rc;
    }
    // output slices one after the other (they share the partial-sum workspace), channel passes within each
    for (int co_lo = 0; co_lo < n_out; co_lo += NO)
    for (int k = 0, lo = 0; lo < c8n; ++k, lo += c8p_max) {
        PsPass Q;
        Q.co_lo = co_lo;
        Q.n_out = n_out;
        Q.c8_lo = lo;
        Q.c8_hi = std::min(c8n, lo + c8p_max);
        Q.part_in = k > 0 ? ws : nullptr;
        Q.part_out = Q.c8_hi < c8n ? ws : nullptr;
        const int c8p = Q.c8_hi - Q.c8_lo;
        const uint32_t cols = ps_tmem_cols(NO, G);
        // deepest ring (group + 1 .. WS_RING_MAX planes) that keeps the CTAs per SM the tensor memory allows
        int ring = 0, best_res = 0;
        size_t smem = 0;
        for (int r = G + 1; r <= WS_RING_MAX && ps_smem_bytes(NO, c8p, r) <= 200 * 1024; ++r) {
            int res = 1;
            const int rc = resident_ctas(conv_ps_kernel<NO, G>, (size_t)ps_smem_bytes(NO, c8p, r) + 1024, cols, res);
            if (rc != CCU_OK) return rc;
            if (res >= best_res) best_res = res, ring = r;
        }
        if (ring == 0) return set_error(CCU_E_INVALID, "plane-stationary pass does not fit shared memory");
        int rc = tc_launch_smem(conv_ps_kernel<NO, G>, ps_smem_bytes(NO, c8p, ring), cols, smem);
        if (rc != CCU_OK) return rc;
        int resident = 1;
        if ((rc = resident_ctas(conv_ps_kernel<NO, G>, smem, cols, resident)) != CCU_OK) return rc;
        const long long grid = std::min<long long>(planes, (long long)sms * resident);
        conv_ps_kernel<NO, G><<<(unsigned)grid, THREADS, smem, st>>>(P, Q, ring);
        CU_CHECK(cudaGetLastError());
    }
    return CCU_OK;
}

// The requested issue group (by default 1: for 16 output channels one chain
// on each of two CTAs per SM measured 1.4x faster than three interleaved
// chains on one CTA), down to the largest whose regions fit 512
// tensor-memory columns (1 for 32 output channels).
template <int NO>
int launch_conv_ps(const ConvP& P, int n_out, int passes, cudaStream_t st) {
    const int group = g_conv_group > 0 ? g_conv_group : 1;
    if (NO == 16 && group == 3) return launch_conv_ps_g<16, 3>(P, n_out, passes, st);
    if (NO == 16 && group == 2) return launch_conv_ps_g<16, 2>(P, n_out, passes, st);
    return launch_conv_ps_g<NO, 1>(P, n_out, passes, st);
}

template <int N>
int launch_conv_halo(const ConvP& P, cudaStream_t st) {
    const int cin = P.src.ca + P.src.cb;
    size_t smem = 0;
    int rc = tc_launch_smem(conv_halo_kernel<N>, halo_smem_bytes(N, cin), tmem_cols(N), smem);
    if (rc != CCU_OK) return rc;
    const long long blocks = (long long)P.src.B * P.src.D * (P.src.H / 16) * (P.src.W / 8);
    conv_halo_kernel<N><<<(unsigned)blocks, THREADS, smem, st>>>(P);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

template <int N>
int launch_wgrad(const WgradP& P, int slices, int cin, cudaStream_t st) {
    size_t smem = 0;
    int rc = tc_launch_smem(wgrad_kernel<N>, (size_t)wgrad_stages(N) * wgrad_stage_bytes(N), tmem_cols(N), smem);
    if (rc != CCU_OK) return rc;
    dim3 grid((unsigned)((27 * cin + TILE_M - 1) / TILE_M), (unsigned)slices);
    wgrad_kernel<N><<<grid, THREADS, smem, st>>>(P);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

// cuTensorMapEncodeTiled from the driver (the runtime is linked statically,
// the driver API is reached through its entry point).
using TensorMapEncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                       const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                       CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

TensorMapEncodeFn tensor_map_encoder() {
    static std::once_flag once;
    static TensorMapEncodeFn fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (TensorMapEncodeFn)p;
    });
    return fn;
}

// 5D map of a [batch][d][h][w][c] BF16 tensor with boxes {bc, bx, by, 1, 1}
// (bc = 16, 32 or 64 channels: rows of 32, 64 or 128 bytes, written with the
// swizzle of that width); coordinates outside it read zeros.
int volume_map(CUtensorMap* m, const void* base, int c, int batch, int d, int h, int w, int bc, int bx, int by) {
    TensorMapEncodeFn enc = tensor_map_encoder();
    if (!enc) return set_error(CCU_E_DEVICE, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[5] = {(cuuint64_t)c, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)d, (cuuint64_t)batch};
    const cuuint64_t strides[4] = {(cuuint64_t)c * 2, (cuuint64_t)w * c * 2, (cuuint64_t)h * w * c * 2,
                                   (cuuint64_t)d * h * w * c * 2};
    const cuuint32_t box[5] = {(cuuint32_t)bc, (cuuint32_t)bx, (cuuint32_t)by, 1u, 1u};
    const cuuint32_t estride[5] = {1u, 1u, 1u, 1u, 1u};
    const CUtensorMapSwizzle sw = bc == 16 ? CU_TENSOR_MAP_SWIZZLE_32B
                                           : (bc == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B);
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(base), dims, strides, box,
                           estride, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(CCU_E_INVALID, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return CCU_OK;
}

template <int N>
int launch_wgrad_tma(const void* a, int ca, int batch, int d, int h, int w, const void* dz, float* dw, int ld,
                     int c_off, int slices, cudaStream_t st) {
    int bx = KSTAGE;
    while (w % bx) bx >>= 1;                        // >= 8: checked by the caller
    const int by = KSTAGE / bx;
    const int a_ch = std::min(ca, 64);             // ca: 16, 32 or a multiple of 64, checked by the caller
    CUtensorMap xmap, zmap;
    int rc = volume_map(&xmap, a, ca, batch, d, h, w, a_ch, bx, by);
    if (rc == CCU_OK) rc = volume_map(&zmap, dz, N, batch, d, h, w, std::min(N, 64), bx, by);
    if (rc != CCU_OK) return rc;
    WgradT P;
    P.dw = dw;
    P.ld = ld;
    P.c_off = c_off;
    P.cin = ca;
    P.rows = 27 * ca;
    P.a_ch = a_ch;
    P.D = d;
    P.bx = bx;
    P.by = by;
    P.nx_blk = w / bx;
    P.ny_blk = (h + by - 1) / by;
    P.stages = (long long)batch * d * P.ny_blk * P.nx_blk;
    size_t smem = 0;
    rc = tc_launch_smem(wgrad_tma_kernel<N>, (size_t)wgrad_tma_stages(N) * wgrad_stage_bytes(N) + 1024, tmem_cols(N),
                        smem);
    if (rc != CCU_OK) return rc;
    // at least four CTAs per SM over the M tiles when the stages allow it
    // (the deep levels have few voxels), else the caller's split
    const int mtiles = (P.rows + TILE_M - 1) / TILE_M;
    const long long want = std::max<long long>(slices, (4LL * sm_count() + mtiles - 1) / mtiles);
    const long long splits = std::max(1LL, std::min<long long>(want, P.stages));
    dim3 grid((unsigned)mtiles, (unsigned)splits);
    wgrad_tma_kernel<N><<<grid, THREADS, smem, st>>>(xmap, zmap, P);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

int g_wgrad_path = 0;       // 0: tile loads where they apply, 1: the gathering kernel

int check_src(const void* a, int ca, const void* b, int cb, int batch, int d, int h, int w) {
    if (!a || ca <= 0 || ca % 16 || cb < 0 || cb % 16 || (cb > 0 && !b))
        return set_error(CCU_E_INVALID, "channels must be positive multiples of 16 (the second input optional)");
    if (!aligned16(a) || (b && !aligned16(b))) return set_error(CCU_E_INVALID, "tensors must be 16-byte aligned");
    if (batch <= 0 || d <= 0 || h <= 0 || w <= 0) return set_error(CCU_E_INVALID, "empty volume");
    if (cb > 0 && (d % 2 || h % 2 || w % 2)) return set_error(CCU_E_INVALID, "upsampled input needs even dimensions");
    if ((long long)batch * d * h * w >= (1LL << 31) - (long long)2 * h * w - 2 * w - 2)
        return set_error(CCU_E_INVALID, "volume too large for 32-bit voxel indices");
    return CCU_OK;
}

}  // namespace

extern "C" {

int ccu_version(void) { return CCU_VERSION; }

const char* ccu_last_error(void) { return t_err.c_str(); }

int ccu_status(unsigned* status, int reset) {
    if (!status) return set_error(CCU_E_INVALID, "NULL argument");
    CU_CHECK(cudaMemcpyFromSymbol(status, g_status, sizeof(unsigned)));
    if (reset) {
        unsigned z = 0;
        CU_CHECK(cudaMemcpyToSymbol(g_status, &z, sizeof(unsigned)));
    }
    return CCU_OK;
}

int ccu_conv3d(const void* a, int ca, const void* b, int cb, int batch, int d, int h, int w, const void* weight,
               const float* bias, int cout, int relu, void* out0, int split, const void* mask0, void* out1,
               void* stream) {
    int rc = check_src(a, ca, b, cb, batch, d, h, w);
    if (rc != CCU_OK) return rc;
    if (!weight || !out0 || split <= 0 || split > cout || split % 8 || (split < cout && !out1))
        return set_error(CCU_E_INVALID, "bad output description");
    if (!aligned16(weight) || !aligned16(out0) || (out1 && !aligned16(out1)) || (mask0 && !aligned16(mask0)))
        return set_error(CCU_E_INVALID, "tensors must be 16-byte aligned");
    ConvP P;
    P.src = Src{(const __nv_bfloat16*)a, (const __nv_bfloat16*)b, ca, cb, batch, d, h, w};
    P.w = (const __nv_bfloat16*)weight;
    P.bias = bias;
    P.relu = relu;
    P.n_vox = (long long)batch * d * h * w;
    P.out0 = (__nv_bfloat16*)out0;
    P.mask0 = (const __nv_bfloat16*)mask0;
    P.split = split;
    P.out1 = (__nv_bfloat16*)out1;
    P.head = nullptr;
    P.head_x = nullptr;
    P.head_out = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    if (const int passes = ps_passes(cout, ca + cb)) {
        if (ps_slice(cout) == 16) return launch_conv_ps<16>(P, cout, passes, st);
        return launch_conv_ps<32>(P, cout, passes, st);
    }
    if (stream_applies(P, cout)) {
        switch (cout) {
            case 16: return launch_conv_stream<16>(P, st);
            case 32: return launch_conv_stream<32>(P, st);
            case 48: return launch_conv_stream<48>(P, st);
            default: break;
        }
    }
    if (halo_applies(P, cout)) {
        switch (cout) {
            case 16: return launch_conv_halo<16>(P, st);
            case 32: return launch_conv_halo<32>(P, st);
            case 48: return launch_conv_halo<48>(P, st);
            default: break;
        }
    }
    switch (cout) {
        case 16: return launch_conv<16>(P, st);
        case 32: return launch_conv<32>(P, st);
        case 48: return launch_conv<48>(P, st);
        case 64: return launch_conv<64>(P, st);
        case 96: return launch_conv<96>(P, st);
        case 128: return launch_conv<128>(P, st);
        case 192: return launch_conv<192>(P, st);
        default: return set_error(CCU_E_INVALID, "output channels must be one of 16, 32, 48, 64, 96, 128, 192");
    }
}

int ccu_conv3d_head(const void* a, int ca, int batch, int d, int h, int w, const void* weight, const float* bias,
                    const float* head, const float* xlog, float* out, void* act, int store_act, void* stream) {
    int rc = check_src(a, ca, nullptr, 0, batch, d, h, w);
    if (rc != CCU_OK) return rc;
    if (!weight || !head || !xlog || !out || (store_act && !act))
        return set_error(CCU_E_INVALID, "bad fused-head arguments");
    if (!aligned16(weight) || (act && !aligned16(act))) return set_error(CCU_E_INVALID, "tensors must be 16-byte aligned");
    const long long n_vox = (long long)batch * d * h * w;
    cudaStream_t st = (cudaStream_t)stream;
    if (ps_passes(16, ca) == 1) {
        ConvP P;
        P.src = Src{(const __nv_bfloat16*)a, nullptr, ca, 0, batch, d, h, w};
        P.w = (const __nv_bfloat16*)weight;
        P.bias = bias;
        P.relu = 1;
        P.n_vox = n_vox;
        P.out0 = store_act ? (__nv_bfloat16*)act : nullptr;
        P.mask0 = nullptr;
        P.split = 16;
        P.out1 = nullptr;
        P.head = head;
        P.head_x = xlog;
        P.head_out = out;
        return launch_conv_ps<16>(P, 16, 1, st);
    }
    // not fusable (another convolution path): the convolution into act, then the head kernel
    if (!act) return set_error(CCU_E_INVALID, "the activation buffer is needed when the head is not fused");
    rc = ccu_conv3d(a, ca, nullptr, 0, batch, d, h, w, weight, bias, 16, 1, act, 16, nullptr, nullptr, stream);
    if (rc != CCU_OK) return rc;
    return ccu_head(act, xlog, nullptr, nullptr, head, 0.0f, n_vox, out, nullptr, nullptr, nullptr, stream);
}

int ccu_conv3d_wgrad(const void* a, int ca, const void* b, int cb, int batch, int d, int h, int w, const void* dz,
                     int cout, float* dw, int slices, void* stream) {
    int rc = check_src(a, ca, b, cb, batch, d, h, w);
    if (rc != CCU_OK) return rc;
    if (!dz || !dw || !aligned16(dz) || slices <= 0) return set_error(CCU_E_INVALID, "bad gradient arguments");
    cudaStream_t st = (cudaStream_t)stream;
    auto box_channels = [](int c) { return c == 16 || c == 32 || c % 64 == 0; };
    if (g_wgrad_path == 0 && w % 8 == 0 && box_channels(ca) && (cb == 0 || box_channels(cb))) {
        if (cout != 16 && cout != 32 && cout != 64 && cout != 128)
            return set_error(CCU_E_INVALID, "output channels must be one of 16, 32, 64, 128");
        auto run = [&](const void* x, int cx, int c_off) {
            switch (cout) {
                case 16: return launch_wgrad_tma<16>(x, cx, batch, d, h, w, dz, dw, ca + cb, c_off, slices, st);
                case 32: return launch_wgrad_tma<32>(x, cx, batch, d, h, w, dz, dw, ca + cb, c_off, slices, st);
                case 64: return launch_wgrad_tma<64>(x, cx, batch, d, h, w, dz, dw, ca + cb, c_off, slices, st);
                default: return launch_wgrad_tma<128>(x, cx, batch, d, h, w, dz, dw, ca + cb, c_off, slices, st);
            }
        };
        if (cb == 0) return run(a, ca, 0);
        // a concatenated layer: the skip part from a, the upsampled part
        // from its full-resolution copy in a per-device buffer
        void* up = nullptr;
        const long long n_vox = (long long)batch * d * h * w;
        rc = grow_buffer(g_up_ws, (size_t)n_vox * cb * 2, st, up);
        if (rc != CCU_OK) return rc;
        upsample_kernel<<<grid_for(n_vox * (cb / 8), 256), 256, 0, st>>>((const uint4*)b, (uint4*)up, batch, d, h, w,
                                                                        cb / 8);
        CU_CHECK(cudaGetLastError());
        rc = run(a, ca, 0);
        if (rc != CCU_OK) return rc;
        return run(up, cb, ca);
    }
    WgradP P;
    P.src = Src{(const __nv_bfloat16*)a, (const __nv_bfloat16*)b, ca, cb, batch, d, h, w};
    P.dz = (const __nv_bfloat16*)dz;
    P.n_vox = (long long)batch * d * h * w;
    long long per = (P.n_vox + slices - 1) / slices;
    per = (per + KSTAGE - 1) / KSTAGE * KSTAGE;
    P.vox_per_cta = per;
    slices = (int)((P.n_vox + per - 1) / per);
    P.dw = dw;
    const int cin = ca + cb;
    switch (cout) {
        case 16: return launch_wgrad<16>(P, slices, cin, st);
        case 32: return launch_wgrad<32>(P, slices, cin, st);
        case 64: return launch_wgrad<64>(P, slices, cin, st);
        case 128: return launch_wgrad<128>(P, slices, cin, st);
        default: return set_error(CCU_E_INVALID, "output channels must be one of 16, 32, 64, 128");
    }
}

int ccu_bias_grad(const void* dz, long long n_vox, int c, float* db, void* stream) {
    if (!dz || !db || c <= 0 || 256 % c) return set_error(CCU_E_INVALID, "bias gradient needs c dividing 256");
    bias_grad_kernel<<<grid_for(n_vox * c, 256), 256, c * sizeof(float), (cudaStream_t)stream>>>(
        (const __nv_bfloat16*)dz, n_vox, c, db);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

int ccu_avgpool(const void* x, int batch, int d, int h, int w, int c, void* y, void* stream) {
    if (!x || !y || c % 8 || d % 2 || h % 2 || w % 2) return set_error(CCU_E_INVALID, "bad pooling arguments");
    long long work = (long long)batch * (d / 2) * (h / 2) * (w / 2) * (c / 8);
    avgpool_kernel<<<grid_for(work, 256), 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)x, batch, d, h, w, c,
                                                                          (__nv_bfloat16*)y);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

int ccu_pool_backward(const void* gy, const void* x_act, int batch, int d, int h, int w, int c, void* dz_x,
                      void* stream) {
    if (!gy || !x_act || !dz_x || c % 8 || d % 2 || h % 2 || w % 2)
        return set_error(CCU_E_INVALID, "bad pooling arguments");
    long long work = (long long)batch * d * h * w * (c / 8);
    pool_backward_kernel<<<grid_for(work, 256), 256, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16*)gy, (const __nv_bfloat16*)x_act, batch, d, h, w, c, (__nv_bfloat16*)dz_x);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

int ccu_up_reduce(const void* g_full, const void* coarse_act, int batch, int d, int h, int w, int c, void* dz_coarse,
                  void* stream) {
    if (!g_full || !coarse_act || !dz_coarse || c % 8 || d % 2 || h % 2 || w % 2)
        return set_error(CCU_E_INVALID, "bad upsampling arguments");
    long long work = (long long)batch * (d / 2) * (h / 2) * (w / 2) * (c / 8);
    up_reduce_kernel<<<grid_for(work, 256), 256, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16*)g_full, (const __nv_bfloat16*)coarse_act, batch, d, h, w, c, (__nv_bfloat16*)dz_coarse);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

int ccu_head(const void* d0, const float* xlog, const float* target, const float* weight, const float* head,
             float inv_wsum, long long n_vox, float* out, void* dz, float* dhead, float* loss, void* stream) {
    if (!d0 || !xlog || !head || (dz && (!target || !dhead))) return set_error(CCU_E_INVALID, "bad head arguments");
    head_kernel<<<grid_for(n_vox, 256), 256, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16*)d0, xlog, target, weight, head, inv_wsum, n_vox, out, (__nv_bfloat16*)dz, dhead, loss);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

int ccu_input(const float* xlog, const float* density, const uint8_t* mat, int n_mat, const float* unc,
              long long n_vox, void* x, void* stream) {
    if (!xlog || !density || !mat || !x || n_mat > 13) return set_error(CCU_E_INVALID, "bad input arguments");
    input_kernel<<<grid_for(n_vox, 256), 256, 0, (cudaStream_t)stream>>>(xlog, density, mat, n_mat, unc, n_vox,
                                                                         (__nv_bfloat16*)x);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

int ccu_adam(float* p, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
             int step, float wd, void* stream) {
    if (!p || !g || !m || !v || step < 1) return set_error(CCU_E_INVALID, "bad optimizer arguments");
    const float c1 = 1.0f / (1.0f - powf(b1, (float)step)), c2 = 1.0f / (1.0f - powf(b2, (float)step));
    adam_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2, wd,
                                                                     nullptr);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

int ccu_adam_clipped(float* p, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                     float eps, int step, float wd, double* clip_state, float clip_ratio, void* stream) {
    if (!p || !g || !m || !v || step < 1 || !clip_state || !(clip_ratio >= 1.0f))
        return set_error(CCU_E_INVALID, "bad optimizer arguments");
    cudaStream_t st = (cudaStream_t)stream;
    const float c1 = 1.0f / (1.0f - powf(b1, (float)step)), c2 = 1.0f / (1.0f - powf(b2, (float)step));
    CU_CHECK(cudaMemsetAsync(clip_state, 0, sizeof(double), st));
    sumsq_kernel<<<(unsigned)std::min<long long>(grid_for(n, 256), 2 * 148), 256, 0, st>>>(g, n, clip_state);
    clip_scale_kernel<<<1, 1, 0, st>>>(clip_state, clip_ratio);
    adam_kernel<<<grid_for(n, 256), 256, 0, st>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2, wd, clip_state);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

long long ccu_packed_weight_elems(int n, int c) {
    if (n <= 0 || c <= 0 || n % 16 || c % 16) return set_error(CCU_E_INVALID, "channels must be positive multiples of 16");
    return packed_elems(n, c);
}

int ccu_pack_weights(const float* w32, int cout, int cin, void* w, void* wt, void* stream) {
    if (!w32 || !w || cout <= 0 || cin <= 0 || cout % 16 || cin % 16)
        return set_error(CCU_E_INVALID, "bad weight arguments");
    const long long total = packed_elems(cout, cin) + (wt ? packed_elems(cin, cout) : 0);
    pack_weights_kernel<<<grid_for(total, 256), 256, 0, (cudaStream_t)stream>>>(w32, cout, cin, (__nv_bfloat16*)w,
                                                                                (__nv_bfloat16*)wt);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

int ccu_set_conv_path(int path) {
    if (path < 0 || path > 4)
        return set_error(CCU_E_INVALID, "path must be 0 (plane-stationary, else streaming, else gathering kernel), "
                                        "1 (gathering kernel), 2 (one-tile halo kernel where it applies), 3 (the "
                                        "streaming kernel with warp roles) or 4 (path 0 without the "
                                        "plane-stationary kernel)");
    g_conv_path = path;
    return CCU_OK;
}

int ccu_set_wgrad_path(int path) {
    if (path < 0 || path > 1)
        return set_error(CCU_E_INVALID, "path must be 0 (tile loads where they apply) or 1 (the gathering kernel)");
    g_wgrad_path = path;
    return CCU_OK;
}

int ccu_set_conv_ring(int ring) {
    if (ring != 0 && (ring < 4 || ring > WS_RING_MAX))
        return set_error(CCU_E_INVALID, "ring must be 0 (chosen per layer) or 4 .. 12 planes");
    g_conv_ring = ring;
    return CCU_OK;
}

int ccu_set_conv_group(int group) {
    if (group < 0 || group > PS_GROUP_MAX)
        return set_error(CCU_E_INVALID, "group must be 0 (chosen per layer) or 1 .. 3 planes");
    g_conv_group = group;
    return CCU_OK;
}

int ccu_zero(void* p, long long bytes, void* stream) {
    if (!p || bytes < 0) return set_error(CCU_E_INVALID, "bad zero arguments");
    CU_CHECK(cudaMemsetAsync(p, 0, (size_t)bytes, (cudaStream_t)stream));
    return CCU_OK;
}

int ccu_gemm_test(const void* a, const void* b, float* d, int m, int n, int k, int a_mn, int b_mn, void* stream) {
    if (!a || !b || !d || m <= 0 || m % TILE_M || n < 16 || n > 256 || n % 16 || k <= 0 || k % 64)
        return set_error(CCU_E_INVALID, "gemm test sizes: m % 128, 16 <= n <= 256 with n % 16, k % 64");
    const size_t smem = (size_t)(TILE_M + n) * 64 * 2;
    // one CTA per SM at most: 256 tensor-memory columns each
    const size_t floor_smem = 120 * 1024;
    const size_t use = smem < floor_smem ? floor_smem : smem;
    CU_CHECK(cudaFuncSetAttribute(gemm_test_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)use));
    gemm_test_kernel<<<m / TILE_M, THREADS, use, (cudaStream_t)stream>>>((const __nv_bfloat16*)a,
                                                                         (const __nv_bfloat16*)b, d, m, n, k, a_mn, b_mn);
    CU_CHECK(cudaGetLastError());
    return CCU_OK;
}

}  // extern "C"
