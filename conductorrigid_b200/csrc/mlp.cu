// mlp.cu -- the per-bead network of the learned initial guess, on the 5th-generation
// tensor cores (tcgen05, BF16 operands, FP32 accumulators in tensor memory).
//
// Network: 48 input features -> 128 (GELU) -> 128 (GELU) -> 1.
//   Z1 = X W1^T, H1 = gelu(Z1 + b1), Z2 = H1 W2^T, y = w3 . gelu(Z2 + b2) + b3.
// Loss (training): (1/n) sum_rows (y - t)^2.
//
// One CTA of 128 threads processes tiles of 128 rows; thread r owns row r of the tile,
// which is TMEM lane r of every M=128 accumulator.  Thread 0 issues the MMAs and
// commits them to one mbarrier; all threads wait on it (bounded by clock64) before
// reading TMEM.  Operands live in shared memory in the canonical K-major, no-swizzle
// layout: 16-byte chunk (row r, k-chunk c) of an R-row operand at byte (c*R + r)*16, so
// the descriptor's leading byte offset (K direction) is R*16 and its stride byte offset
// (8-row groups) is 128.
//
// The training kernel runs forward and backward per tile:
//   MMA1  Z1     = X    . W1^T            (TMEM cols   0..127)
//   MMA2  Z2     = H1   . W2^T            (TMEM cols 128..255)
//   MMA3  dH1    = dZ2  . W2              (TMEM cols 128..255, over Z2)
//   MMA4  dW2ext += dZ2^T . [H1 | 1]      (TMEM cols 256..399: dW2 and, col 128, db2)
//   MMA5  dW1ext += dZ1^T . [X  | 1]      (TMEM cols 400..463: dW1 and, col 48, db1)
// The ones row appended to the transposed B operands turns the bias gradients into
// one more accumulator column.  Weight gradients stay in TMEM across a CTA's tiles and
// are added to the global FP32 gradient once per CTA.  dZ2 and dZ1 are rounded to BF16
// for the MMAs (the CPU check rounds at the same points).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/conductor_rigid.h"

namespace crmlp {

constexpr int F = CR_MLP_FEATURES;   // 48
constexpr int H = CR_MLP_HIDDEN;     // 128
constexpr int TM = 128;              // rows per tile
constexpr int FX = F + 16;           // X^T with the ones row (rows 48..63)
constexpr int HX = H + 16;           // H1^T with the ones row (rows 128..143)

// parameter offsets in the flat FP32 vector
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + H * F;
constexpr int OFF_W2 = OFF_B1 + H;
constexpr int OFF_B2 = OFF_W2 + H * H;
constexpr int OFF_W3 = OFF_B2 + H;
constexpr int OFF_B3 = OFF_W3 + H;
constexpr int NPARAM = OFF_B3 + 1;
static_assert(NPARAM == CR_MLP_PARAMS, "parameter count");

// TMEM column map
constexpr uint32_t TC_Z1 = 0, TC_Z2 = 128, TC_DW2 = 256, TC_DW1 = 400;

// shared memory map (bytes); sizes of K-major operands are rows * k * 2
constexpr int SZ_W2 = H * H * 2, SZ_HD = TM * H * 2, SZ_H1T = HX * TM * 2, SZ_DZ2T = H * TM * 2;
constexpr int SZ_X = TM * F * 2, SZ_W1 = H * F * 2, SZ_XT = FX * TM * 2;

// Farthest byte one MMA chain can address from an operand's base: the start of its last
// K step plus the span of one descriptor, taken as the larger of the two readings of the
// strides (K chunks at R*16 or at 128 bytes, 8-row groups at 128 or at R*16 bytes).  The
// allocation is padded to the largest reach, so no descriptor can address past it.
constexpr int reach(int base, int rows, int k) {
    return base + (k / 16 - 1) * 2 * rows * 16 + (rows / 8 - 1) * rows * 16 + rows * 16 + 256;
}
constexpr int cmax(int a, int b) { return a > b ? a : b; }

struct TrainLayout {
    static constexpr int w2 = 0, w2t = w2 + SZ_W2, hd = w2t + SZ_W2, h1t = hd + SZ_HD, dz2t = h1t + SZ_H1T,
                         x = dz2t + SZ_DZ2T, w1 = x + SZ_X, xt = w1 + SZ_W1, vec = xt + SZ_XT,
                         // fp32 b1, b2, w3, dw3 (4 x 128) then the mbarrier and the TMEM address
                         bar = vec + 4 * H * 4, taddr = bar + 8, end = taddr + 8;
    static constexpr int bytes =
        cmax(end, cmax(cmax(reach(hd, TM, H), reach(h1t, HX, TM)),
                       cmax(cmax(reach(dz2t, H, TM), reach(x, TM, F)), cmax(reach(w1, H, F), reach(xt, FX, TM)))));
};
struct InferLayout {
    static constexpr int w2 = 0, hd = w2 + SZ_W2, x = hd + SZ_HD, w1 = x + SZ_X, vec = w1 + SZ_W1,
                         bar = vec + 4 * H * 4, taddr = bar + 8, end = taddr + 8;
    static constexpr int bytes = cmax(end, cmax(cmax(reach(hd, TM, H), reach(x, TM, F)), reach(w1, H, F)));
};
static_assert(TrainLayout::bytes <= 227 * 1024, "training kernel shared memory");
static_assert(InferLayout::bytes <= 227 * 1024, "inference kernel shared memory");

// ---- PTX wrappers ----------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr, uint32_t rows) {
    const uint64_t lbo = (uint64_t)rows * 16u;  // next 8-element K chunk
    const uint64_t sbo = 128u;                  // next group of 8 rows
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | (((lbo >> 4) & 0x3FFFull) << 16) | (((sbo >> 4) & 0x3FFFull) << 32) |
           (1ull << 46);  // descriptor version 1, base offset 0, no swizzle
}

// BF16 x BF16 -> FP32, both operands K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Wait for the barrier phase `parity` to complete; gives up after `limit` cycles (2^31 by
// default, about a second) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit) {
    const uint32_t a = smem_u32(bar);
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > limit) return false;
    }
}

// ---- activation --------------------------------------------------------------------
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&v);
}
__device__ __forceinline__ uint16_t bf16_bits(float a) {
    __nv_bfloat16 v = __float2bfloat16_rn(a);
    return *reinterpret_cast<uint16_t *>(&v);
}

// byte offset of element (row r, column k) in a K-major operand of R rows
__device__ __forceinline__ int kofs(int r, int k, int R) { return ((k >> 3) * R + r) * 16 + (k & 7) * 2; }

// W (rows x k, row-major FP32) -> K-major BF16 operand
__device__ void stage_weight(uint8_t *dst, const float *W, int rows, int k) {
    for (int c = threadIdx.x; c < rows * (k / 8); c += blockDim.x) {
        const int r = c % rows, kc = c / rows;
        const float *w = W + (size_t)r * k + kc * 8;
        uint4 v;
        v.x = pack2(w[0], w[1]);
        v.y = pack2(w[2], w[3]);
        v.z = pack2(w[4], w[5]);
        v.w = pack2(w[6], w[7]);
        *reinterpret_cast<uint4 *>(dst + (kc * rows + r) * 16) = v;
    }
}

struct Accum {
    float loss = 0.f, db3 = 0.f;
};

// Issue `ksteps` K=16 MMAs A(rowsA) x B(rowsB)^T into dtmem.
__device__ __forceinline__ void mma_chain(uint32_t dtmem, uint32_t a, uint32_t rows_a, uint32_t b, uint32_t rows_b,
                                          uint32_t n, int ksteps, bool accumulate) {
    const uint32_t idesc = idesc_bf16(n);
    for (int kk = 0; kk < ksteps; ++kk)
        mma_bf16(dtmem, kmajor_desc(a + kk * 2 * rows_a * 16, rows_a), kmajor_desc(b + kk * 2 * rows_b * 16, rows_b),
                 idesc, (accumulate || kk > 0) ? 1u : 0u);
}

template <bool TRAIN>
__global__ void __launch_bounds__(128, 1)
    mlp_kernel(int n, const uint16_t *__restrict__ X, const float *__restrict__ target, float inv_n,
               const float *__restrict__ params, float *__restrict__ y_out, float *__restrict__ grad,
               float *__restrict__ stats, int *__restrict__ err, long long wait_limit, int withhold_first) {
    extern __shared__ __align__(1024) uint8_t smem[];
    using Lay = typename std::conditional<TRAIN, TrainLayout, InferLayout>::type;
    constexpr uint32_t NCOL = TRAIN ? 512 : 256;  // one CTA per SM (shared memory)
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + Lay::bar);
    uint32_t *taddr_s = reinterpret_cast<uint32_t *>(smem + Lay::taddr);
    float *b1s = reinterpret_cast<float *>(smem + Lay::vec);
    float *b2s = b1s + H, *w3s = b2s + H, *dw3s = w3s + H;
    const uint32_t s_base = smem_u32(smem);

    if (warp == 0) tmem_alloc(taddr_s, NCOL);
    if (tid == 0) mbar_init(bar);
    stage_weight(smem + Lay::w1, params + OFF_W1, H, F);
    stage_weight(smem + Lay::w2, params + OFF_W2, H, H);
    for (int i = tid; i < H; i += blockDim.x) {
        b1s[i] = params[OFF_B1 + i];
        b2s[i] = params[OFF_B2 + i];
        w3s[i] = params[OFF_W3 + i];
        dw3s[i] = 0.f;
    }
    const float b3 = params[OFF_B3];
    if constexpr (TRAIN) {
        // W2^T: element (in, out) = W2[out][in]
        uint8_t *w2t = smem + TrainLayout::w2t;
        for (int c = tid; c < H * (H / 8); c += blockDim.x) {
            const int r = c % H, kc = c / H;
            const float *w = params + OFF_W2 + r;
            uint4 v;
            v.x = pack2(w[(kc * 8 + 0) * H], w[(kc * 8 + 1) * H]);
            v.y = pack2(w[(kc * 8 + 2) * H], w[(kc * 8 + 3) * H]);
            v.z = pack2(w[(kc * 8 + 4) * H], w[(kc * 8 + 5) * H]);
            v.w = pack2(w[(kc * 8 + 6) * H], w[(kc * 8 + 7) * H]);
            *reinterpret_cast<uint4 *>(w2t + (kc * H + r) * 16) = v;
        }
        // ones rows of the transposed operands (row 48 of X^T, row 128 of H1^T), zeros after
        for (int s = tid; s < TM; s += blockDim.x) {
            for (int r = F; r < FX; ++r)
                *reinterpret_cast<uint16_t *>(smem + TrainLayout::xt + kofs(r, s, FX)) = r == F ? 0x3F80 : 0;
            for (int r = H; r < HX; ++r)
                *reinterpret_cast<uint16_t *>(smem + TrainLayout::h1t + kofs(r, s, HX)) = r == H ? 0x3F80 : 0;
        }
    }
    async_fence();
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tm = *taddr_s;
    const uint32_t lane_tm = tm + ((uint32_t)(warp * 32) << 16);
    uint32_t phase = 0;
    bool failed = false;
    Accum acc;
    const int ntiles = (n + TM - 1) / TM;
    int done_tiles = 0;

    auto sync_wait = [&]() -> bool {
        const bool ok = mbar_wait(bar, phase, wait_limit);
        phase ^= 1u;
        tc_after();
        return __syncthreads_or(!ok) == 0;
    };
    auto handoff = [&]() {  // threads' smem writes and TMEM reads done before the next MMA
        async_fence();
        tc_before();
        __syncthreads();
    };

    for (int tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
        const int row = tile * TM + tid;
        const bool valid = row < n;
        // ---- stage X (and X^T) ----
        uint4 xr[F / 8];
#pragma unroll
        for (int c = 0; c < F / 8; ++c)
            xr[c] = valid ? *reinterpret_cast<const uint4 *>(X + (size_t)row * F + c * 8) : make_uint4(0, 0, 0, 0);
#pragma unroll
        for (int c = 0; c < F / 8; ++c) *reinterpret_cast<uint4 *>(smem + Lay::x + (c * TM + tid) * 16) = xr[c];
        if constexpr (TRAIN) {
            const uint16_t *xe = reinterpret_cast<const uint16_t *>(xr);
#pragma unroll
            for (int f = 0; f < F; ++f)
                *reinterpret_cast<uint16_t *>(smem + TrainLayout::xt + kofs(f, tid, FX)) = xe[f];
        }
        handoff();
        // ---- MMA1: Z1 = X W1^T ----
        // (withhold_first: a test hook that issues neither these MMAs nor their commit on the
        // CTA's first tile, so nothing arrives on the barrier and its bounded wait runs out
        // with no tensor-core work in flight)
        if (tid == 0 && !(withhold_first && tile == (int)blockIdx.x)) {
            tc_after();
            mma_chain(tm + TC_Z1, s_base + Lay::x, TM, s_base + Lay::w1, H, H, F / 16, false);
            mma_commit(bar);
        }
        if (!sync_wait()) { failed = true; break; }
        // ---- H1 = gelu(Z1 + b1) -> BF16 operands ----
        for (int c0 = 0; c0 < H; c0 += 16) {
            float v[16];
            tmem_ld16(lane_tm + TC_Z1 + c0, v);
            uint32_t p[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) p[j] = pack2(gelu(v[2 * j] + b1s[c0 + 2 * j]), gelu(v[2 * j + 1] + b1s[c0 + 2 * j + 1]));
            *reinterpret_cast<uint4 *>(smem + Lay::hd + kofs(tid, c0, TM)) = make_uint4(p[0], p[1], p[2], p[3]);
            *reinterpret_cast<uint4 *>(smem + Lay::hd + kofs(tid, c0 + 8, TM)) = make_uint4(p[4], p[5], p[6], p[7]);
            if constexpr (TRAIN) {
                const uint16_t *pe = reinterpret_cast<const uint16_t *>(p);
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    *reinterpret_cast<uint16_t *>(smem + TrainLayout::h1t + kofs(c0 + j, tid, HX)) = pe[j];
            }
        }
        handoff();
        // ---- MMA2: Z2 = H1 W2^T ----
        if (tid == 0) {
            tc_after();
            mma_chain(tm + TC_Z2, s_base + Lay::hd, TM, s_base + Lay::w2, H, H, H / 16, false);
            mma_commit(bar);
        }
        if (!sync_wait()) { failed = true; break; }
        float y = b3;
        for (int c0 = 0; c0 < H; c0 += 16) {
            float v[16];
            tmem_ld16(lane_tm + TC_Z2 + c0, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) y += w3s[c0 + j] * gelu(v[j] + b2s[c0 + j]);
        }
        if constexpr (!TRAIN) {
            if (valid) y_out[row] = y;
            tc_before();
            __syncthreads();
            ++done_tiles;
            continue;
        } else {
            const float e = valid ? y - target[row] : 0.f;
            const float dy = 2.f * e * inv_n;
            acc.loss += e * e;
            acc.db3 += dy;
            // ---- dZ2 = dy w3 gelu'(Z2 + b2); dw3 += dy h2 ----
            for (int c0 = 0; c0 < H; c0 += 16) {
                float v[16];
                tmem_ld16(lane_tm + TC_Z2 + c0, v);
                uint32_t p[8];
#pragma unroll
                for (int j = 0; j < 16; j += 2) {
                    const float a0 = v[j] + b2s[c0 + j], a1 = v[j + 1] + b2s[c0 + j + 1];
                    p[j / 2] = pack2(dy * w3s[c0 + j] * gelu_grad(a0), dy * w3s[c0 + j + 1] * gelu_grad(a1));
                    float s0 = dy * gelu(a0), s1 = dy * gelu(a1);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
                        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
                    }
                    if (lane == 0) {
                        atomicAdd(&dw3s[c0 + j], s0);
                        atomicAdd(&dw3s[c0 + j + 1], s1);
                    }
                }
                *reinterpret_cast<uint4 *>(smem + TrainLayout::hd + kofs(tid, c0, TM)) = make_uint4(p[0], p[1], p[2], p[3]);
                *reinterpret_cast<uint4 *>(smem + TrainLayout::hd + kofs(tid, c0 + 8, TM)) =
                    make_uint4(p[4], p[5], p[6], p[7]);
                const uint16_t *pe = reinterpret_cast<const uint16_t *>(p);
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    *reinterpret_cast<uint16_t *>(smem + TrainLayout::dz2t + kofs(c0 + j, tid, H)) = pe[j];
            }
            handoff();
            // ---- MMA3: dH1 = dZ2 W2;  MMA4: [dW2 | db2] += dZ2^T [H1 | 1] ----
            if (tid == 0) {
                tc_after();
                mma_chain(tm + TC_Z2, s_base + TrainLayout::hd, TM, s_base + TrainLayout::w2t, H, H, H / 16, false);
                mma_chain(tm + TC_DW2, s_base + TrainLayout::dz2t, H, s_base + TrainLayout::h1t, HX, HX, TM / 16,
                          done_tiles > 0);
                mma_commit(bar);
            }
            if (!sync_wait()) { failed = true; break; }
            // ---- dZ1 = dH1 gelu'(Z1 + b1) -> dZ1^T ----
            for (int c0 = 0; c0 < H; c0 += 16) {
                float g[16], z[16];
                tmem_ld16(lane_tm + TC_Z2 + c0, g);
                tmem_ld16(lane_tm + TC_Z1 + c0, z);
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    *reinterpret_cast<uint16_t *>(smem + TrainLayout::hd + kofs(c0 + j, tid, H)) =
                        bf16_bits(g[j] * gelu_grad(z[j] + b1s[c0 + j]));
            }
            handoff();
            // ---- MMA5: [dW1 | db1] += dZ1^T [X | 1] ----
            if (tid == 0) {
                tc_after();
                mma_chain(tm + TC_DW1, s_base + TrainLayout::hd, H, s_base + TrainLayout::xt, FX, FX, TM / 16,
                          done_tiles > 0);
                mma_commit(bar);
            }
            if (!sync_wait()) { failed = true; break; }
            ++done_tiles;
        }
    }

    if constexpr (TRAIN) {
        if (!failed && done_tiles > 0) {
            // thread r holds output unit r of both weight-gradient accumulators
            for (int c0 = 0; c0 < HX; c0 += 16) {
                float v[16];
                tmem_ld16(lane_tm + TC_DW2 + c0, v);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int c = c0 + j;
                    if (c < H) atomicAdd(&grad[OFF_W2 + tid * H + c], v[j]);
                    else if (c == H) atomicAdd(&grad[OFF_B2 + tid], v[j]);
                }
            }
            for (int c0 = 0; c0 < FX; c0 += 16) {
                float v[16];
                tmem_ld16(lane_tm + TC_DW1 + c0, v);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int c = c0 + j;
                    if (c < F) atomicAdd(&grad[OFF_W1 + tid * F + c], v[j]);
                    else if (c == F) atomicAdd(&grad[OFF_B1 + tid], v[j]);
                }
            }
            __syncthreads();
            atomicAdd(&grad[OFF_W3 + tid], dw3s[tid]);
            float l = acc.loss, d3 = acc.db3;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                l += __shfl_xor_sync(0xffffffffu, l, o);
                d3 += __shfl_xor_sync(0xffffffffu, d3, o);
            }
            if (lane == 0) {
                atomicAdd(&stats[0], l);
                atomicAdd(&grad[OFF_B3], d3);
            }
        }
    }
    if (failed && tid == 0) atomicExch(err, 1);
    tc_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tm, NCOL);
}

__global__ void adam_kernel(int np, float *__restrict__ p, float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                            float clip) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    float gi = fminf(fmaxf(g[i], -clip), clip);
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    g[i] = 0.f;
}

}  // namespace crmlp

struct cr_mlp {
    int device = 0;
    int n_sm = 148;
    float *d_param = nullptr, *d_grad = nullptr, *d_m = nullptr, *d_v = nullptr, *d_stats = nullptr;
    int *d_err = nullptr;
    long long wait_limit = 1ll << 31;  // clock cycles of every bounded barrier wait
    int withhold_first = 0;            // test hook: the next launch withholds its first MMAs
    long long adam_steps = 0;
    long long launches = 0;
    std::string last_error;
};

namespace {

int mlp_fail(cr_mlp *h, int st, const std::string &msg) {
    if (h) h->last_error = msg;
    return st;
}
int mlp_cuda(cr_mlp *h, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return CR_OK;
    cudaGetLastError();
    return mlp_fail(h, e == cudaErrorMemoryAllocation ? CR_OUT_OF_MEMORY : CR_CUDA_ERROR,
                    std::string(what) + ": " + cudaGetErrorString(e));
}
#define MLP_CUDA(h, expr)                                   \
    do {                                                    \
        int _st = mlp_cuda((h), (expr), #expr);             \
        if (_st != CR_OK) return _st;                       \
    } while (0)

bool g_attr_done[64] = {};
std::mutex g_attr_mu;

int set_attrs(cr_mlp *h) {
    std::lock_guard<std::mutex> lk(g_attr_mu);
    if (h->device < 64 && g_attr_done[h->device]) return CR_OK;
    MLP_CUDA(h, cudaFuncSetAttribute(crmlp::mlp_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     crmlp::TrainLayout::bytes));
    MLP_CUDA(h, cudaFuncSetAttribute(crmlp::mlp_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     crmlp::InferLayout::bytes));
    if (h->device < 64) g_attr_done[h->device] = true;
    return CR_OK;
}

int check_err(cr_mlp *h, cudaStream_t s) {
    int e = 0;
    MLP_CUDA(h, cudaMemcpyAsync(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    MLP_CUDA(h, cudaStreamSynchronize(s));
    if (e) {
        MLP_CUDA(h, cudaMemsetAsync(h->d_err, 0, sizeof(int), s));
        return mlp_fail(h, CR_TIMEOUT, "tensor-core wait ran out");
    }
    return CR_OK;
}

}  // namespace

namespace cr {

// Inference without the host-side error check (for use inside a solve, also while a
// stream is being captured): the kernel records a wait that ran out in the network's
// error flag, which mlp_check reads later.
int mlp_forward_async(cr_mlp *h, int n, const uint16_t *d_x, float *d_y, cudaStream_t s) {
    if (!h || n <= 0) return CR_OK;
    const int ntiles = (n + crmlp::TM - 1) / crmlp::TM;
    const int grid = std::min(ntiles, h->n_sm);
    crmlp::mlp_kernel<false><<<grid, 128, crmlp::InferLayout::bytes, s>>>(n, d_x, nullptr, 0.f, h->d_param, d_y,
                                                                            nullptr, nullptr, h->d_err,
                                                                            h->wait_limit, 0);
    ++h->launches;
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CR_OK : CR_CUDA_ERROR;
}

// CR_TIMEOUT if a wait of an earlier asynchronous launch ran out (clears the flag).
int mlp_check(cr_mlp *h, cudaStream_t s) { return check_err(h, s); }

}  // namespace cr

extern "C" {

int cr_mlp_create(uint64_t seed, cr_mlp **out) {
    if (!out) return CR_BAD_PARAM;
    *out = nullptr;
    cr_mlp *h = new cr_mlp();
    int st = CR_OK;
    auto fail_out = [&](int s) {
        cr_mlp_destroy(h);
        return s;
    };
    if ((st = mlp_cuda(h, cudaGetDevice(&h->device), "cudaGetDevice")) != CR_OK) return fail_out(st);
    cudaDeviceProp prop;
    if ((st = mlp_cuda(h, cudaGetDeviceProperties(&prop, h->device), "cudaGetDeviceProperties")) != CR_OK)
        return fail_out(st);
    if (prop.major != 10) return fail_out(mlp_fail(h, CR_BAD_PARAM, "the tensor-core network needs an sm_100 GPU"));
    h->n_sm = prop.multiProcessorCount;
    const size_t bytes = crmlp::NPARAM * sizeof(float);
    for (float **p : {&h->d_param, &h->d_grad, &h->d_m, &h->d_v})
        if ((st = mlp_cuda(h, cudaMalloc((void **)p, bytes), "cudaMalloc")) != CR_OK) return fail_out(st);
    if ((st = mlp_cuda(h, cudaMalloc((void **)&h->d_stats, 4 * sizeof(float)), "cudaMalloc")) != CR_OK ||
        (st = mlp_cuda(h, cudaMalloc((void **)&h->d_err, sizeof(int)), "cudaMalloc")) != CR_OK)
        return fail_out(st);
    // He-style initialisation from a SplitMix64 stream (host), biases zero
    std::vector<float> p(crmlp::NPARAM, 0.f);
    uint64_t z = seed;
    auto uni = [&]() {
        z += 0x9E3779B97F4A7C15ull;
        uint64_t x = z;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        x ^= x >> 31;
        return (double)(x >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    const double s1 = std::sqrt(3.0 / crmlp::F), s2 = std::sqrt(3.0 / crmlp::H);
    for (int i = 0; i < crmlp::H * crmlp::F; ++i) p[crmlp::OFF_W1 + i] = (float)(s1 * uni());
    for (int i = 0; i < crmlp::H * crmlp::H; ++i) p[crmlp::OFF_W2 + i] = (float)(s2 * uni());
    for (int i = 0; i < crmlp::H; ++i) p[crmlp::OFF_W3 + i] = (float)(0.1 * s2 * uni());
    if ((st = mlp_cuda(h, cudaMemcpy(h->d_param, p.data(), bytes, cudaMemcpyHostToDevice), "cudaMemcpy")) != CR_OK)
        return fail_out(st);
    for (float *q : {h->d_grad, h->d_m, h->d_v})
        if ((st = mlp_cuda(h, cudaMemset(q, 0, bytes), "cudaMemset")) != CR_OK) return fail_out(st);
    if ((st = mlp_cuda(h, cudaMemset(h->d_stats, 0, 4 * sizeof(float)), "cudaMemset")) != CR_OK ||
        (st = mlp_cuda(h, cudaMemset(h->d_err, 0, sizeof(int)), "cudaMemset")) != CR_OK)
        return fail_out(st);
    if ((st = set_attrs(h)) != CR_OK) return fail_out(st);
    *out = h;
    return CR_OK;
}

int cr_mlp_destroy(cr_mlp *h) {
    if (!h) return CR_BAD_PARAM;
    for (float *p : {h->d_param, h->d_grad, h->d_m, h->d_v, h->d_stats})
        if (p) cudaFree(p);
    if (h->d_err) cudaFree(h->d_err);
    delete h;
    return CR_OK;
}

const char *cr_mlp_last_error(const cr_mlp *h) { return h ? h->last_error.c_str() : "null network"; }

int cr_mlp_get_params(cr_mlp *h, float *params) {
    if (!h || !params) return CR_BAD_PARAM;
    MLP_CUDA(h, cudaMemcpy(params, h->d_param, crmlp::NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    return CR_OK;
}

int cr_mlp_set_params(cr_mlp *h, const float *params) {
    if (!h || !params) return CR_BAD_PARAM;
    MLP_CUDA(h, cudaMemcpy(h->d_param, params, crmlp::NPARAM * sizeof(float), cudaMemcpyHostToDevice));
    return CR_OK;
}

int cr_mlp_get_grads(cr_mlp *h, float *grads) {
    if (!h || !grads) return CR_BAD_PARAM;
    MLP_CUDA(h, cudaMemcpy(grads, h->d_grad, crmlp::NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    return CR_OK;
}

int cr_mlp_forward(cr_mlp *h, int n, const uint16_t *d_x, float *d_y, void *stream) {
    if (!h || n < 0 || (n > 0 && (!d_x || !d_y))) return mlp_fail(h, CR_BAD_PARAM, "bad forward arguments");
    if ((uintptr_t)d_x % 16) return mlp_fail(h, CR_BAD_PARAM, "features must be 16-byte aligned");
    if (n == 0) return CR_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int ntiles = (n + crmlp::TM - 1) / crmlp::TM;
    const int grid = std::min(ntiles, h->n_sm);
    crmlp::mlp_kernel<false><<<grid, 128, crmlp::InferLayout::bytes, s>>>(n, d_x, nullptr, 0.f, h->d_param, d_y,
                                                                            nullptr, nullptr, h->d_err,
                                                                            h->wait_limit, h->withhold_first);
    h->withhold_first = 0;
    ++h->launches;
    MLP_CUDA(h, cudaGetLastError());
    return check_err(h, s);
}

int cr_mlp_accumulate_grad(cr_mlp *h, int n, const uint16_t *d_x, const float *d_t, double *loss, void *stream) {
    if (!h || n < 0 || (n > 0 && (!d_x || !d_t))) return mlp_fail(h, CR_BAD_PARAM, "bad training arguments");
    if ((uintptr_t)d_x % 16) return mlp_fail(h, CR_BAD_PARAM, "features must be 16-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    MLP_CUDA(h, cudaMemsetAsync(h->d_stats, 0, 4 * sizeof(float), s));
    if (n > 0) {
        const int ntiles = (n + crmlp::TM - 1) / crmlp::TM;
        const int grid = std::min(ntiles, h->n_sm);
        crmlp::mlp_kernel<true><<<grid, 128, crmlp::TrainLayout::bytes, s>>>(n, d_x, d_t, 1.f / n, h->d_param,
                                                                               nullptr, h->d_grad, h->d_stats, h->d_err,
                                                                               h->wait_limit, h->withhold_first);
        h->withhold_first = 0;
        ++h->launches;
        MLP_CUDA(h, cudaGetLastError());
    }
    int st = check_err(h, s);
    if (st != CR_OK) return st;
    if (loss) {
        float l = 0.f;
        MLP_CUDA(h, cudaMemcpy(&l, h->d_stats, sizeof(float), cudaMemcpyDeviceToHost));
        *loss = n > 0 ? (double)l / n : 0.0;
    }
    return CR_OK;
}

int cr_mlp_adam(cr_mlp *h, double lr, double clip, void *stream) {
    if (!h || !(lr > 0.0) || !(clip > 0.0)) return mlp_fail(h, CR_BAD_PARAM, "bad optimiser arguments");
    const double b1 = 0.9, b2 = 0.999;
    ++h->adam_steps;
    const double c1 = 1.0 - std::pow(b1, (double)h->adam_steps), c2 = 1.0 - std::pow(b2, (double)h->adam_steps);
    crmlp::adam_kernel<<<(crmlp::NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        crmlp::NPARAM, h->d_param, h->d_grad, h->d_m, h->d_v, (float)lr, (float)b1, (float)b2, 1e-8f, (float)c1,
        (float)c2, (float)clip);
    ++h->launches;
    MLP_CUDA(h, cudaGetLastError());
    return CR_OK;
}

int cr_mlp_set_wait(cr_mlp *h, long long max_cycles, int withhold_next) {
    if (!h || max_cycles < 1000) return mlp_fail(h, CR_BAD_PARAM, "wait limit below 1000 cycles");
    h->wait_limit = max_cycles;
    h->withhold_first = withhold_next ? 1 : 0;
    return CR_OK;
}

int cr_mlp_counters(const cr_mlp *h, long long *kernel_launches, long long *adam_steps) {
    if (!h || !kernel_launches || !adam_steps) return CR_BAD_PARAM;
    *kernel_launches = h->launches;
    *adam_steps = h->adam_steps;
    return CR_OK;
}

}  // extern "C"
