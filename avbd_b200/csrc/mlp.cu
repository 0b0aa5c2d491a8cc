// mlp.cu -- the learned warm start's multilayer perceptron on the tensor
// cores: a generic BF16 GEMM (training), the fused persistent inference
// kernel (the hot path: features -> 4 layers -> x0 update), and the training
// kernels (bias + SiLU, loss, activation gradient, transposes, Adam).
//
// The reference has no learned component; this is new functionality.  All
// matrix products run as tcgen05.mma (kind::f16, BF16 operands in shared
// memory, FP32 accumulators in tensor memory).
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include "engine.h"
#include "tc05.cuh"

using bf16 = __nv_bfloat16;

namespace avbd {
namespace {

constexpr unsigned HID = AVBD_MLP_HIDDEN;    // 128
constexpr unsigned IN = AVBD_MLP_IN_PAD;     // 32
constexpr unsigned OUT = AVBD_MLP_OUT_PAD;   // 16
// offsets of the flat parameter array
constexpr unsigned OFF_W1 = 0, OFF_B1 = 4096, OFF_W2 = 4224, OFF_B2 = 20608, OFF_W3 = 20736, OFF_B3 = 37120,
                   OFF_W4 = 37248, OFF_B4 = 39296, NPAR = AVBD_MLP_NPARAMS;
static_assert(OFF_B1 == HID * IN && OFF_W2 == OFF_B1 + HID && OFF_B2 == OFF_W2 + HID * HID &&
                  OFF_W3 == OFF_B2 + HID && OFF_B3 == OFF_W3 + HID * HID && OFF_W4 == OFF_B3 + HID &&
                  OFF_B4 == OFF_W4 + OUT * HID && NPAR == OFF_B4 + OUT,
              "parameter layout");

AVBD_D float silu(float z) { return z / (1.0f + __expf(-z)); }
// The same function as z/2 (1 + tanh(z/2)) with the hardware tanh
// approximation (one special-function operation instead of two; its error,
// about 2^-11 relative, is below the BF16 rounding of the result).
AVBD_D float silu_fast(float z) {
    const float h = 0.5f * z;
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(h));
    return fmaf(h, t, h);
}
AVBD_D float silu_grad(float z) {
    float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}
AVBD_D uint32_t pack2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

// R x K row-major BF16 global matrix (row stride ld) -> K-major canonical
// shared layout; rows >= rows_valid are zero
AVBD_D void load_kmaj(uint8_t* dst, const bf16* src, unsigned ld, unsigned R, unsigned K, unsigned rows_valid,
                      unsigned tid, unsigned nthreads) {
    const unsigned pieces = R * (K / 8);
    for (unsigned i = tid; i < pieces; i += nthreads) {
        const unsigned r = i % R, c = i / R;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (r < rows_valid) v = __ldg(reinterpret_cast<const uint4*>(src + (size_t)r * ld + c * 8));
        *reinterpret_cast<uint4*>(dst + c * (R * 16) + r * 16) = v;
    }
}

// Polls a barrier wait may take before it gives up (avbd_debug_set_wait_limit
// lowers it so that tests can make the wait run out).
__device__ uint32_t g_wait_polls = AVBD_DEFAULT_WAIT_POLLS;
// Polls the drain after a timeout may take: the MMAs already issued must
// land before the CTA frees the TMEM columns they write.
constexpr uint32_t kDrainPolls = AVBD_DEFAULT_WAIT_POLLS;

// all threads wait for the barrier phase; false (uniformly) if it timed out
AVBD_D bool block_wait(uint64_t* bar, uint32_t& phase) {
    bool got = tc::mbar_wait(bar, phase, *(volatile uint32_t*)&g_wait_polls);
    phase ^= 1u;
    return __syncthreads_and(got ? 1 : 0) != 0;
}

// After a wait gave up (phase already flipped by block_wait): wait, bounded,
// for the commit of the MMAs still in flight, so that no tensor-core write
// reaches the TMEM columns after they are freed.
AVBD_D void drain_after_timeout(uint64_t* bar, uint32_t phase) {
    if (threadIdx.x == 0) tc::mbar_wait(bar, phase ^ 1u, kDrainPolls);
    __syncthreads();
}

// one thread: D (+)= A B^T over `ksteps` K = 16 steps of two canonical operands
AVBD_D void issue(uint32_t d, uint32_t a, uint32_t a_rows, uint32_t b, uint32_t b_rows, unsigned ksteps,
                  uint32_t idesc, bool acc_first) {
    for (unsigned s = 0; s < ksteps; s++) {
        uint64_t da = tc::sdesc(a + s * 2 * a_rows * 16, a_rows * 16, 128);
        uint64_t db = tc::sdesc(b + s * 2 * b_rows * 16, b_rows * 16, 128);
        tc::mma_bf16(d, da, db, idesc, (acc_first || s > 0) ? 1u : 0u);
    }
}

// ------------------------------------------------------------ generic GEMM
// C [M x N] (+)= A [M x K] B [N x K]^T.  One CTA: 128 rows x NT columns, a
// K range of `kper` (split-K over blockIdx.z, atomics when split), K chunks
// of 64 staged in shared memory.
template <int NT>
__global__ void __launch_bounds__(128) k_gemm(const bf16* __restrict__ A, unsigned lda, const bf16* __restrict__ B,
                                              unsigned ldb, float* C, unsigned ldc, unsigned M, unsigned N, unsigned K,
                                              unsigned kper, int mode, int* err) {
    __shared__ __align__(1024) uint8_t sA[128 * 64 * 2];
    __shared__ __align__(1024) uint8_t sB[NT * 64 * 2];
    __shared__ uint64_t bar;
    __shared__ uint32_t tslot;
    constexpr uint32_t TCOLS = NT < 32 ? 32 : NT;
    const unsigned tid = threadIdx.x, warp = tid >> 5;
    const unsigned row0 = blockIdx.x * 128, col0 = blockIdx.y * NT;
    const unsigned kb = blockIdx.z * kper, ke = min(K, kb + kper);
    if (warp == 0) tc::tmem_alloc(&tslot, TCOLS);
    if (tid == 0) tc::mbar_init(&bar, 1);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = tslot;
    const uint32_t idesc = tc::idesc_bf16(128, NT);
    const unsigned mrows = M > row0 ? min(128u, M - row0) : 0u;
    const unsigned nrows = N > col0 ? min((unsigned)NT, N - col0) : 0u;
    uint32_t phase = 0;
    bool ok = true;
    for (unsigned k0 = kb; k0 < ke && ok; k0 += 64) {
        const unsigned kl = min(64u, ke - k0);  // a multiple of 16
        load_kmaj(sA, A + (size_t)row0 * lda + k0, lda, 128, kl, mrows, tid, 128);
        load_kmaj(sB, B + (size_t)col0 * ldb + k0, ldb, NT, kl, nrows, tid, 128);
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after();
            issue(tmem, tc::smem_u32(sA), 128, tc::smem_u32(sB), NT, kl / 16, idesc, k0 > kb);
            tc::commit(&bar);
        }
        ok = block_wait(&bar, phase);
    }
    if (!ok) drain_after_timeout(&bar, phase);
    tc::fence_after();
    if (ok && ke > kb) {
        const unsigned r = warp * 32 + (tid & 31);
        const unsigned gr = row0 + r;
#pragma unroll
        for (unsigned c = 0; c < (unsigned)NT; c += 16) {
            float v[16];
            tc::tmem_ld16(tmem + ((warp * 32u) << 16) + c, v);
            if (gr < M) {
                float* dst = C + (size_t)gr * ldc + col0 + c;
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    if (col0 + c + j >= N) break;
                    if (mode == 0) dst[j] = v[j];
                    else if (mode == 1) dst[j] += v[j];
                    else atomicAdd(dst + j, v[j]);
                }
            }
        }
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::tmem_dealloc(tmem, TCOLS);
        tc::tmem_relinquish();
    }
    if (!ok && tid == 0) atomicExch(err, (int)AVBD_ERR_BARRIER_TIMEOUT);
}

}  // namespace

// C = A B^T (+ C): tile width from N, split-K when there are too few tiles
int gemm_bf16(const bf16* A, unsigned lda, const bf16* B, unsigned ldb, float* C, unsigned ldc, unsigned M,
              unsigned N, unsigned K, bool accumulate, cudaStream_t st, int* err) {
    if (M == 0 || N == 0 || K == 0) return AVBD_OK;
    if (K % 16 || lda % 8 || ldb % 8 || ((uintptr_t)A & 15) || ((uintptr_t)B & 15))
        return set_error(AVBD_ERR_INVALID_ARG, "gemm: K % 16, lda % 8, ldb % 8 and 16-byte aligned operands required");
    const unsigned NT = N <= 16 ? 16 : (N <= 32 ? 32 : 128);
    const unsigned mt = (M + 127) / 128, nt = (N + NT - 1) / NT;
    unsigned split = 1;
    if (mt * nt < 148 && K >= 512) split = std::min(K / 256, std::max(1u, 148u / (mt * nt)));
    unsigned kper = ((K + split - 1) / split + 63) / 64 * 64;
    split = (K + kper - 1) / kper;
    int mode = accumulate ? 1 : 0;
    if (split > 1) {  // partial sums are added atomically into a zeroed C
        if (!accumulate) {
            cudaError_t e = cudaMemset2DAsync(C, sizeof(float) * ldc, 0, sizeof(float) * N, M, st);
            if (e != cudaSuccess) return set_error(AVBD_ERR_CUDA, cudaGetErrorString(e));
        }
        mode = 2;
    }
    dim3 grid(mt, nt, split);
    if (NT == 16) k_gemm<16><<<grid, 128, 0, st>>>(A, lda, B, ldb, C, ldc, M, N, K, kper, mode, err);
    else if (NT == 32) k_gemm<32><<<grid, 128, 0, st>>>(A, lda, B, ldb, C, ldc, M, N, K, kper, mode, err);
    // 128-column tiles: 15 KB of unused dynamic shared memory caps residency at
    // 4 CTAs per SM, so their TMEM (4 x 128 columns) always fits at once
    else k_gemm<128><<<grid, 128, 15360, st>>>(A, lda, B, ldb, C, ldc, M, N, K, kper, mode, err);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? AVBD_OK : set_error(AVBD_ERR_CUDA, cudaGetErrorString(e));
}

// ------------------------------------------------------ fused inference
namespace {

struct MlpW {
    const bf16 *w1, *w2, *w3, *w4;
    const float* b;  // b1 | b2 | b3 | b4 (400 floats)
};

// Where the outputs go: a plain FP32 array (out != null) or the solver
// state (x0 += scale * y for internal vertex `row`, with the iteration
// history x_last / x_lastlast reset to the new guess).
template <typename P>
struct MlpSink {
    float* out;
    typename Vec4Of<P>::T *x, *xl, *xll;
    const uint8_t* flags;  // row = internal vertex; fixed and oriented vertices are skipped
    P scale;
    float kappa;           // relative error assumed by the acceptance test
    unsigned long long* applied;  // count of accepted corrections (may be null)
};

constexpr unsigned SM_W1 = 0, SM_W2 = 8192, SM_W3 = 40960, SM_W4 = 73728, SM_X = 77824, SM_H = 94208,
                   SM_BIAS = 126976, SM_BAR = 128576, SM_TSLOT = 128584, SM_TOTAL = 128640;  // X: 2 x 8 KB

// Feature tile (128 rows x 32 BF16) -> canonical K-major shared layout with
// cp.async (rows >= rows_valid are zero-filled), so the next tile streams in
// while this one runs through the layers.
AVBD_D void load_x_async(uint8_t* dst, const bf16* src, unsigned rows_valid, unsigned tid) {
    for (unsigned i = tid; i < 128 * (IN / 8); i += blockDim.x) {
        const unsigned r = i % 128, c = i / 128;
        const bool in = r < rows_valid;
        const bf16* g = in ? src + (size_t)r * IN + c * 8 : src;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(tc::smem_u32(dst + c * (128 * 16) + r * 16)),
                     "l"(g), "r"(in ? 16 : 0)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// TMEM accumulator -> bias + SiLU -> BF16 into the H operand.  16 warps:
// warp w reads lanes 32 (w % 4).. (rows) and the column quarter w / 4 (16
// warps rather than 8: 4 % less time per launch, the epilogue being
// latency-bound).
AVBD_D void epilogue_hidden(uint32_t tacc, const float* bias, uint8_t* H, unsigned warp, unsigned lane) {
    const unsigned q = warp & 3u, hf = warp >> 2;  // 16 warps: column quarters
    const unsigned r = q * 32 + lane;
    const uint32_t base = tacc + ((q * 32u) << 16);
#pragma unroll
    for (unsigned c = hf * 32; c < hf * 32 + 32; c += 16) {
        float v[16];
        tc::tmem_ld16(base + c, v);
        uint32_t pk[8];
#pragma unroll
        for (int j = 0; j < 8; j++)
            pk[j] = pack2(silu_fast(v[2 * j] + bias[c + 2 * j]), silu_fast(v[2 * j + 1] + bias[c + 2 * j + 1]));
        *reinterpret_cast<uint4*>(H + (c / 8) * (128 * 16) + r * 16) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        *reinterpret_cast<uint4*>(H + (c / 8 + 1) * (128 * 16) + r * 16) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
    }
}

// Acceptance of the correction y (in units of s = g h^2) of one vertex.  The
// block residual at the inertial guess is r0 = |features 12-14| (units of
// m g, L1).  Applying y with a relative error kappa leaves a residual of
// about kappa * sum_a (1 + H_aa h^2 / m) |y_a| (features 18-20 hold
// log(1 + H_aa h^2 / m)), so the correction is applied only where it removes
// more residual than its error adds, and never below 1e-4 m g (a vertex in
// free flight, where the inertial guess is exact up to rounding).
constexpr float WS_GATE = 1e-4f;
AVBD_D bool accept(const uint8_t* Xs, unsigned r, const float* y, float kappa) {
    const bf16* f = reinterpret_cast<const bf16*>(Xs + tc::kmaj_off(r, 12, 128));
    const bf16* h = reinterpret_cast<const bf16*>(Xs + tc::kmaj_off(r, 16, 128));  // features 16..23
    const float r0 = fabsf(__bfloat162float(f[0])) + fabsf(__bfloat162float(f[1])) + fabsf(__bfloat162float(f[2]));
    const float added = kappa * (__expf(__bfloat162float(h[2])) * fabsf(y[0]) +
                                 __expf(__bfloat162float(h[3])) * fabsf(y[1]) +
                                 __expf(__bfloat162float(h[4])) * fabsf(y[2]));
    return r0 > WS_GATE && r0 > added;
}

// Persistent: one CTA per SM, weights resident in shared memory, 128 feature
// rows per tile; layers alternate between TMEM columns [0,128) and [128,256).
template <typename P>
__global__ void __launch_bounds__(512, 1) k_mlp_apply(MlpW w, const bf16* __restrict__ feat, unsigned n,
                                                       MlpSink<P> sink, int* err) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t* W1s = sm + SM_W1;
    uint8_t* W2s = sm + SM_W2;
    uint8_t* W3s = sm + SM_W3;
    uint8_t* W4s = sm + SM_W4;
    uint8_t* Xbuf = sm + SM_X;  // two 8 KB tiles
    uint8_t* Hs = sm + SM_H;
    float* bias = reinterpret_cast<float*>(sm + SM_BIAS);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + SM_BAR);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + SM_TSLOT);
    const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    load_kmaj(W1s, w.w1, IN, HID, IN, HID, tid, 512);
    load_kmaj(W2s, w.w2, HID, HID, HID, HID, tid, 512);
    load_kmaj(W3s, w.w3, HID, HID, HID, HID, tid, 512);
    load_kmaj(W4s, w.w4, HID, OUT, HID, OUT, tid, 512);
    for (unsigned i = tid; i < 3 * HID + OUT; i += 512) bias[i] = w.b[i];
    if (warp == 0) tc::tmem_alloc(tslot, 256);
    if (tid == 0) tc::mbar_init(bar, 1);
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t accA = tmem, accB = tmem + 128;
    const uint32_t id_h = tc::idesc_bf16(128, HID), id_o = tc::idesc_bf16(128, OUT);
    const uint32_t aH = tc::smem_u32(Hs);
    uint32_t phase = 0;
    bool ok = true;
    const unsigned ntiles = (n + 127) / 128;
    if (blockIdx.x < ntiles) {
        const unsigned r0 = blockIdx.x * 128;
        load_x_async(Xbuf, feat + (size_t)r0 * IN, min(128u, n - r0), tid);
    }
    unsigned buf = 0;
    for (unsigned tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, buf ^= 1u) {
        const unsigned row0 = tile * 128;
        uint8_t* Xs = Xbuf + buf * 8192;
        const uint32_t aX = tc::smem_u32(Xs);
        const unsigned next = tile + gridDim.x;
        if (next < ntiles) {  // the other buffer was last read by the previous tile, finished
            const unsigned r1 = next * 128;
            load_x_async(Xbuf + (buf ^ 1u) * 8192, feat + (size_t)r1 * IN, min(128u, n - r1), tid);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        tc::fence_async_smem();
        __syncthreads();
        // layer 1: X W1^T -> accA
        if (tid == 0) {
            tc::fence_after();
            issue(accA, aX, 128, tc::smem_u32(W1s), HID, IN / 16, id_h, false);
            tc::commit(bar);
        }
        if (!(ok = block_wait(bar, phase))) break;
        tc::fence_after();
        epilogue_hidden(accA, bias, Hs, warp, lane);
        tc::fence_before();
        tc::fence_async_smem();
        __syncthreads();
        // layer 2: H W2^T -> accB
        if (tid == 0) {
            tc::fence_after();
            issue(accB, aH, 128, tc::smem_u32(W2s), HID, HID / 16, id_h, false);
            tc::commit(bar);
        }
        if (!(ok = block_wait(bar, phase))) break;
        tc::fence_after();
        epilogue_hidden(accB, bias + HID, Hs, warp, lane);
        tc::fence_before();
        tc::fence_async_smem();
        __syncthreads();
        // layer 3: H W3^T -> accA
        if (tid == 0) {
            tc::fence_after();
            issue(accA, aH, 128, tc::smem_u32(W3s), HID, HID / 16, id_h, false);
            tc::commit(bar);
        }
        if (!(ok = block_wait(bar, phase))) break;
        tc::fence_after();
        epilogue_hidden(accA, bias + 2 * HID, Hs, warp, lane);
        tc::fence_before();
        tc::fence_async_smem();
        __syncthreads();
        // layer 4: H W4^T -> accB columns [0, 16)
        if (tid == 0) {
            tc::fence_after();
            issue(accB, aH, 128, tc::smem_u32(W4s), OUT, HID / 16, id_o, false);
            tc::commit(bar);
        }
        if (!(ok = block_wait(bar, phase))) break;
        tc::fence_after();
        if (warp < 4) {
            float v[16];
            tc::tmem_ld16(accB + ((warp * 32u) << 16), v);
            const unsigned row = row0 + warp * 32 + lane;
            if (row < n) {
                const float* b4 = bias + 3 * HID;
                if (sink.out) {
#pragma unroll
                    for (int j = 0; j < 16; j++) sink.out[(size_t)row * OUT + j] = v[j] + b4[j];
                } else if (!(sink.flags[row] & (VF_FIXED | VF_ORIENTED))) {
                    const float y[3] = {v[0] + b4[0], v[1] + b4[1], v[2] + b4[2]};
                    if (accept(Xs, warp * 32 + lane, y, sink.kappa)) {
                        if (sink.applied) atomicAdd(sink.applied, 1ull);
                        typename Vec4Of<P>::T x4 = sink.x[row];
                        x4.x += sink.scale * (P)y[0];
                        x4.y += sink.scale * (P)y[1];
                        x4.z += sink.scale * (P)y[2];
                        sink.x[row] = x4;
                        sink.xl[row] = x4;
                        sink.xll[row] = x4;
                    }
                }
            }
        }
        tc::fence_before();
        __syncthreads();
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");  // no copy may land after the exit
    if (!ok) drain_after_timeout(bar, phase);
    tc::fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::tmem_dealloc(tmem, 256);
        tc::tmem_relinquish();
    }
    if (!ok && tid == 0) atomicExch(err, (int)AVBD_ERR_BARRIER_TIMEOUT);
}

// ------------------------------------------------------ training kernels
// Z [B x N] += bias (kept as the pre-activation); H = act(Z) in BF16, both
// row-major [B][N] and transposed [N][B]
__global__ void k_bias_act(float* Z, const float* bias, unsigned B, unsigned N, bool act, bf16* H, bf16* HT) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)B * N) return;
    unsigned r = (unsigned)(i / N), c = (unsigned)(i % N);
    float z = Z[i] + bias[c];
    Z[i] = z;
    float h = act ? silu(z) : z;
    bf16 hb = __float2bfloat16_rn(h);
    if (H) H[i] = hb;
    if (HT) HT[(size_t)c * B + r] = hb;
}

// loss = mean over rows and the 3 outputs of w (y - t)^2, w the row's
// weight (target column 3); dY = dloss/dy in BF16 ([B][16] and [16][B]);
// db4 += column sums
__global__ void k_loss(const float* Y, const float* T, unsigned B, bf16* dY, bf16* dYT, float* loss, float* db4) {
    unsigned r = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0, g[AVBD_MLP_OUT] = {0, 0, 0};
    if (r < B) {
        const float w = T[(size_t)r * 4 + 3];
#pragma unroll
        for (int j = 0; j < (int)OUT; j++) {
            float d = 0;
            if (j < AVBD_MLP_OUT) {
                float e = Y[(size_t)r * OUT + j] - T[(size_t)r * 4 + j];
                l += w * e * e;
                d = 2.0f * w * e / (float)(B * AVBD_MLP_OUT);
                g[j] = d;
            }
            bf16 db = __float2bfloat16_rn(d);
            dY[(size_t)r * OUT + j] = db;
            dYT[(size_t)j * B + r] = db;
        }
    }
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) {
        l += __shfl_xor_sync(0xffffffffu, l, m);
#pragma unroll
        for (int j = 0; j < AVBD_MLP_OUT; j++) g[j] += __shfl_xor_sync(0xffffffffu, g[j], m);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(loss, l / (float)(B * AVBD_MLP_OUT));
        for (int j = 0; j < AVBD_MLP_OUT; j++) atomicAdd(db4 + j, g[j]);
    }
}

// dZ = dH * silu'(Z) in BF16 ([B][N] and [N][B]); db += column sums
__global__ void k_act_grad(const float* dH, const float* Z, unsigned B, unsigned N, bf16* dZ, bf16* dZT, float* db) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)B * N) return;
    unsigned r = (unsigned)(i / N), c = (unsigned)(i % N);
    float d = dH[i] * silu_grad(Z[i]);
    bf16 b = __float2bfloat16_rn(d);
    dZ[i] = b;
    dZT[(size_t)c * B + r] = b;
    atomicAdd(db + c, d);
}

__global__ void k_transpose_bf16(const bf16* src, unsigned R, unsigned Cc, unsigned lds, bf16* dst) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)R * Cc) return;
    unsigned r = (unsigned)(i / Cc), c = (unsigned)(i % Cc);
    dst[(size_t)c * R + r] = src[(size_t)r * lds + c];
}

__global__ void k_transpose_f32(const float* src, unsigned R, unsigned Cc, float* dst) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)R * Cc) return;
    unsigned r = (unsigned)(i / Cc), c = (unsigned)(i % Cc);
    dst[(size_t)c * R + r] = src[i];
}

// master FP32 parameters -> BF16 weights ([out][in] and [in][out]) and FP32
// biases of the four layers
__global__ void k_pack(const float* P, bf16* w1, bf16* w2, bf16* w3, bf16* w4, bf16* w1t, bf16* w2t, bf16* w3t,
                       bf16* w4t, float* b) {
    unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < HID * IN) {
        unsigned o = i / IN, k = i % IN;
        bf16 v = __float2bfloat16_rn(P[OFF_W1 + i]);
        w1[i] = v;
        if (w1t) w1t[k * HID + o] = v;
    }
    if (i < HID * HID) {
        unsigned o = i / HID, k = i % HID;
        bf16 v2 = __float2bfloat16_rn(P[OFF_W2 + i]), v3 = __float2bfloat16_rn(P[OFF_W3 + i]);
        w2[i] = v2;
        w3[i] = v3;
        if (w2t) w2t[k * HID + o] = v2;
        if (w3t) w3t[k * HID + o] = v3;
    }
    if (i < OUT * HID) {
        unsigned o = i / HID, k = i % HID;
        bf16 v = __float2bfloat16_rn(P[OFF_W4 + i]);
        w4[i] = v;
        if (w4t) w4t[k * OUT + o] = v;
    }
    if (i < HID) {
        b[i] = P[OFF_B1 + i];
        b[HID + i] = P[OFF_B2 + i];
        b[2 * HID + i] = P[OFF_B3 + i];
    }
    if (i < OUT) b[3 * HID + i] = P[OFF_B4 + i];
}

// padding that must stay zero: inputs 27..31 of W1, outputs 3..15 of W4 / b4
AVBD_D bool frozen(unsigned i) {
    if (i < OFF_B1) return (i % IN) >= AVBD_MLP_IN;
    if (i >= OFF_W4 && i < OFF_B4) return (i - OFF_W4) / HID >= AVBD_MLP_OUT;
    if (i >= OFF_B4) return i - OFF_B4 >= AVBD_MLP_OUT;
    return false;
}

__global__ void k_adam(float* P, const float* G, float* Mo, float* Vo, float lr, float c1, float c2) {
    unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NPAR || frozen(i)) return;
    float g = G[i];
    float m = 0.9f * Mo[i] + 0.1f * g;
    float v = 0.999f * Vo[i] + 0.001f * g * g;
    Mo[i] = m;
    Vo[i] = v;
    P[i] -= lr * (m / c1) / (sqrtf(v / c2) + 1e-8f);
}

inline unsigned nb(size_t n, unsigned per) { return (unsigned)((n + per - 1) / per); }

}  // namespace

// BF16 weights + FP32 biases of one MLP on the device
struct MlpDevice {
    bf16 *w1 = nullptr, *w2 = nullptr, *w3 = nullptr, *w4 = nullptr;
    float* b = nullptr;
    float* p32 = nullptr;
    int* err = nullptr;
    int device = 0;
    int upload(const float* params, cudaStream_t st);
    void release();
};

int MlpDevice::upload(const float* params, cudaStream_t st) {
    if (!params) return set_error(AVBD_ERR_INVALID_ARG, "null parameters");
    auto al = [](void** p, size_t bytes) { return cudaMalloc(p, bytes); };
    if (!w1) {
        if (al((void**)&w1, sizeof(bf16) * HID * IN) || al((void**)&w2, sizeof(bf16) * HID * HID) ||
            al((void**)&w3, sizeof(bf16) * HID * HID) || al((void**)&w4, sizeof(bf16) * OUT * HID) ||
            al((void**)&b, sizeof(float) * (3 * HID + OUT)) || al((void**)&p32, sizeof(float) * NPAR) ||
            al((void**)&err, sizeof(int)))
            return set_error(AVBD_ERR_CUDA, "MLP weight allocation failed");
        cudaMemsetAsync(err, 0, sizeof(int), st);
    }
    if (cudaMemcpyAsync(p32, params, sizeof(float) * NPAR, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return set_error(AVBD_ERR_CUDA, "MLP parameter upload failed");
    k_pack<<<nb(HID * HID, 256), 256, 0, st>>>(p32, w1, w2, w3, w4, nullptr, nullptr, nullptr, nullptr, b);
    cudaError_t e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? AVBD_OK : set_error(AVBD_ERR_CUDA, cudaGetErrorString(e));
}

void MlpDevice::release() {
    for (void* p : {(void*)w1, (void*)w2, (void*)w3, (void*)w4, (void*)b, (void*)p32, (void*)err})
        if (p) cudaFree(p);
    w1 = w2 = w3 = w4 = nullptr;
    b = p32 = nullptr;
    err = nullptr;
}

static int grid_for(int device, unsigned n) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return (int)std::max(1u, std::min((n + 127) / 128, (unsigned)sms));
}

template <typename P>
static int mlp_launch(const MlpDevice& m, const bf16* feat, unsigned n, const MlpSink<P>& sink, cudaStream_t st) {
    if (n == 0) return AVBD_OK;
    static std::atomic<uint64_t> attr_set[2];  // bit d: set on device d
    std::atomic<uint64_t>& done = attr_set[sizeof(P) == 8];
    const uint64_t bit = 1ull << (m.device & 63);
    if (!(done.load() & bit)) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_apply<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM_TOTAL);
        if (e != cudaSuccess) return set_error(AVBD_ERR_CUDA, cudaGetErrorString(e));
        done.fetch_or(bit);
    }
    MlpW w{m.w1, m.w2, m.w3, m.w4, m.b};
    k_mlp_apply<P><<<grid_for(m.device, n), 512, SM_TOTAL, st>>>(w, feat, n, sink, m.err);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? AVBD_OK : set_error(AVBD_ERR_CUDA, cudaGetErrorString(e));
}

// x0 update of the engine's warm start (rows: internal vertex of each row)
template <typename P>
int mlp_apply_state(const MlpDevice& m, const void* feat, unsigned n, typename Vec4Of<P>::T* x,
                    typename Vec4Of<P>::T* xl, typename Vec4Of<P>::T* xll, const uint8_t* flags, double scale,
                    float kappa, unsigned long long* applied, cudaStream_t st) {
    MlpSink<P> s{nullptr, x, xl, xll, flags, (P)scale, kappa, applied};
    return mlp_launch<P>(m, (const bf16*)feat, n, s, st);
}
template int mlp_apply_state<float>(const MlpDevice&, const void*, unsigned, float4*, float4*, float4*,
                                    const uint8_t*, double, float, unsigned long long*, cudaStream_t);
template int mlp_apply_state<double>(const MlpDevice&, const void*, unsigned, double4a*, double4a*, double4a*,
                                     const uint8_t*, double, float, unsigned long long*, cudaStream_t);

int mlp_device_upload(MlpDevice** m, int device, const float* params, cudaStream_t st) {
    if (!*m) {
        *m = new MlpDevice();
        (*m)->device = device;
    }
    return (*m)->upload(params, st);
}
void mlp_device_free(MlpDevice* m) {
    if (m) {
        m->release();
        delete m;
    }
}
int mlp_device_error(const MlpDevice* m, cudaStream_t st) {
    int h = 0;
    if (!m || !m->err) return AVBD_OK;
    if (cudaMemcpyAsync(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return set_error(AVBD_ERR_CUDA, "MLP error flag read failed");
    if (!h) return AVBD_OK;
    // the flag is cleared once reported, so the object stays usable
    if (cudaMemsetAsync(m->err, 0, sizeof(int), st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
        return set_error(AVBD_ERR_CUDA, "MLP error flag reset failed");
    return set_error(h, "MLP kernel: a bounded wait on the tensor-core barrier gave up; every result of that "
                        "launch is invalid");
}

}  // namespace avbd

using namespace avbd;

// ------------------------------------------------------------------- C-ABI
struct avbd_mlp {
    MlpDevice* m = nullptr;
    cudaStream_t st = nullptr;
};

struct avbd_mlp_trainer {
    int device = 0;
    unsigned B = 0;
    cudaStream_t st = nullptr;
    MlpDevice w;                  // BF16 [out][in] weights + biases
    bf16 *w1t = nullptr, *w2t = nullptr, *w3t = nullptr, *w4t = nullptr;  // [in][out]
    float *G = nullptr, *Mo = nullptr, *Vo = nullptr;
    float *Z1 = nullptr, *Z2 = nullptr, *Z3 = nullptr, *Y = nullptr;      // [B][128] x3, [B][16]
    bf16 *H1 = nullptr, *H2 = nullptr, *H3 = nullptr;                     // [B][128]
    bf16 *H1T = nullptr, *H2T = nullptr, *H3T = nullptr, *XT = nullptr;   // [128][B] x3, [32][B]
    bf16 *dY = nullptr, *dYT = nullptr, *dZ = nullptr, *dZT = nullptr;    // [B][16], [16][B], [B][128], [128][B]
    float *dH = nullptr, *dW4T = nullptr, *loss = nullptr;                // [B][128], [128][16], 1
    unsigned t = 0;
    std::vector<void*> allocs;
};

extern "C" {

int avbd_gemm_bf16(const void* A, unsigned lda, const void* B, unsigned ldb, float* C, unsigned ldc, unsigned M,
                   unsigned N, unsigned K, int accumulate, void* stream) {
    if (!A || !B || !C) return set_error(AVBD_ERR_INVALID_ARG, "null operand");
    int* err = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return set_error(AVBD_ERR_CUDA, "cudaMalloc");
    cudaMemsetAsync(err, 0, sizeof(int), st);
    int rc = gemm_bf16((const bf16*)A, lda, (const bf16*)B, ldb, C, ldc, M, N, K, accumulate != 0, st, err);
    int h = 0;
    cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(err);
    if (rc) return rc;
    if (e != cudaSuccess) return set_error(AVBD_ERR_CUDA, cudaGetErrorString(e));
    return h ? set_error(h, "GEMM: a bounded wait on the tensor-core barrier gave up") : AVBD_OK;
}

int avbd_debug_set_wait_limit(int device, unsigned polls) {
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess)
        return set_error(AVBD_ERR_NO_DEVICE, "cudaSetDevice failed");
    cudaError_t e = cudaMemcpyToSymbol(g_wait_polls, &polls, sizeof(polls));
    int rc = e == cudaSuccess ? solve_set_wait_limit(polls) : AVBD_OK;
    if (e == cudaSuccess && rc == AVBD_OK) rc = contacts_set_wait_limit(polls);
    if (e == cudaSuccess && rc == AVBD_OK) e = cudaDeviceSynchronize();
    cudaSetDevice(prev);
    if (rc != AVBD_OK) return rc;
    return e == cudaSuccess ? AVBD_OK : set_error(AVBD_ERR_CUDA, cudaGetErrorString(e));
}

int avbd_mlp_create(avbd_mlp** out, int device, const float* params) {
    if (!out || !params) return set_error(AVBD_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return set_error(AVBD_ERR_NO_DEVICE, "cudaSetDevice failed");
    avbd_mlp* m = new avbd_mlp();
    cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking);
    if (int rc = mlp_device_upload(&m->m, device, params, m->st)) {
        mlp_device_free(m->m);
        cudaStreamDestroy(m->st);
        delete m;
        return rc;
    }
    *out = m;
    return AVBD_OK;
}

int avbd_mlp_forward(avbd_mlp* m, const void* features, unsigned n, float* out, void* stream) {
    if (!m || !features || !out) return set_error(AVBD_ERR_INVALID_ARG, "null argument");
    if ((uintptr_t)features & 15) return set_error(AVBD_ERR_INVALID_ARG, "features must be 16-byte aligned");
    cudaStream_t st = stream ? (cudaStream_t)stream : m->st;
    MlpSink<float> s{out, nullptr, nullptr, nullptr, nullptr, 0.f, 0.f, nullptr};
    if (int rc = mlp_launch<float>(*m->m, (const bf16*)features, n, s, st)) return rc;
    return mlp_device_error(m->m, st);
}

int avbd_mlp_destroy(avbd_mlp* m) {
    if (!m) return AVBD_OK;
    mlp_device_free(m->m);
    if (m->st) cudaStreamDestroy(m->st);
    delete m;
    return AVBD_OK;
}

int avbd_mlp_trainer_create(avbd_mlp_trainer** out, int device, unsigned batch, const float* params) {
    if (!out || !params) return set_error(AVBD_ERR_INVALID_ARG, "null argument");
    if (batch == 0 || batch % 128) return set_error(AVBD_ERR_INVALID_ARG, "batch must be a positive multiple of 128");
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return set_error(AVBD_ERR_NO_DEVICE, "cudaSetDevice failed");
    auto* t = new avbd_mlp_trainer();
    t->device = device;
    t->B = batch;
    cudaStreamCreateWithFlags(&t->st, cudaStreamNonBlocking);
    const size_t B = batch;
    bool bad = false;
    auto al = [&](auto** p, size_t bytes) {
        if (bad) return;
        if (cudaMalloc((void**)p, bytes) != cudaSuccess) bad = true;
        else t->allocs.push_back((void*)*p);
    };
    al(&t->w1t, sizeof(bf16) * HID * IN); al(&t->w2t, sizeof(bf16) * HID * HID);
    al(&t->w3t, sizeof(bf16) * HID * HID); al(&t->w4t, sizeof(bf16) * OUT * HID);
    al(&t->G, sizeof(float) * NPAR); al(&t->Mo, sizeof(float) * NPAR); al(&t->Vo, sizeof(float) * NPAR);
    al(&t->Z1, sizeof(float) * B * HID); al(&t->Z2, sizeof(float) * B * HID); al(&t->Z3, sizeof(float) * B * HID);
    al(&t->Y, sizeof(float) * B * OUT);
    al(&t->H1, sizeof(bf16) * B * HID); al(&t->H2, sizeof(bf16) * B * HID); al(&t->H3, sizeof(bf16) * B * HID);
    al(&t->H1T, sizeof(bf16) * B * HID); al(&t->H2T, sizeof(bf16) * B * HID); al(&t->H3T, sizeof(bf16) * B * HID);
    al(&t->XT, sizeof(bf16) * B * IN);
    al(&t->dY, sizeof(bf16) * B * OUT); al(&t->dYT, sizeof(bf16) * B * OUT);
    al(&t->dZ, sizeof(bf16) * B * HID); al(&t->dZT, sizeof(bf16) * B * HID);
    al(&t->dH, sizeof(float) * B * HID); al(&t->dW4T, sizeof(float) * HID * OUT); al(&t->loss, sizeof(float));
    if (bad) {
        avbd_mlp_trainer_destroy(t);
        return set_error(AVBD_ERR_CUDA, "trainer allocation failed");
    }
    t->w.device = device;
    if (int rc = t->w.upload(params, t->st)) {
        avbd_mlp_trainer_destroy(t);
        return rc;
    }
    cudaMemsetAsync(t->Mo, 0, sizeof(float) * NPAR, t->st);
    cudaMemsetAsync(t->Vo, 0, sizeof(float) * NPAR, t->st);
    k_pack<<<nb(HID * HID, 256), 256, 0, t->st>>>(t->w.p32, t->w.w1, t->w.w2, t->w.w3, t->w.w4, t->w1t, t->w2t,
                                                  t->w3t, t->w4t, t->w.b);
    if (cudaStreamSynchronize(t->st) != cudaSuccess) {
        avbd_mlp_trainer_destroy(t);
        return set_error(AVBD_ERR_CUDA, "trainer initialisation failed");
    }
    *out = t;
    return AVBD_OK;
}

// forward + backward of one mini-batch into t->G (and t->loss)
static int trainer_fwd_bwd(avbd_mlp_trainer* t, const bf16* X, const float* T) {
    const unsigned B = t->B;
    cudaStream_t st = t->st;
    int* err = t->w.err;
    const float* b = t->w.b;
    int rc;
    cudaMemsetAsync(t->G, 0, sizeof(float) * NPAR, st);
    cudaMemsetAsync(t->loss, 0, sizeof(float), st);
    // forward
    if ((rc = gemm_bf16(X, IN, t->w.w1, IN, t->Z1, HID, B, HID, IN, false, st, err))) return rc;
    k_bias_act<<<nb((size_t)B * HID, 256), 256, 0, st>>>(t->Z1, b, B, HID, true, t->H1, t->H1T);
    if ((rc = gemm_bf16(t->H1, HID, t->w.w2, HID, t->Z2, HID, B, HID, HID, false, st, err))) return rc;
    k_bias_act<<<nb((size_t)B * HID, 256), 256, 0, st>>>(t->Z2, b + HID, B, HID, true, t->H2, t->H2T);
    if ((rc = gemm_bf16(t->H2, HID, t->w.w3, HID, t->Z3, HID, B, HID, HID, false, st, err))) return rc;
    k_bias_act<<<nb((size_t)B * HID, 256), 256, 0, st>>>(t->Z3, b + 2 * HID, B, HID, true, t->H3, t->H3T);
    if ((rc = gemm_bf16(t->H3, HID, t->w.w4, HID, t->Y, OUT, B, OUT, HID, false, st, err))) return rc;
    k_bias_act<<<nb((size_t)B * OUT, 256), 256, 0, st>>>(t->Y, b + 3 * HID, B, OUT, false, nullptr, nullptr);
    k_transpose_bf16<<<nb((size_t)B * IN, 256), 256, 0, st>>>(X, B, IN, IN, t->XT);
    // loss and output layer
    k_loss<<<nb(B, 256), 256, 0, st>>>(t->Y, T, B, t->dY, t->dYT, t->loss, t->G + OFF_B4);
    if ((rc = gemm_bf16(t->H3T, B, t->dYT, B, t->dW4T, OUT, HID, OUT, B, false, st, err))) return rc;
    k_transpose_f32<<<nb(HID * OUT, 256), 256, 0, st>>>(t->dW4T, HID, OUT, t->G + OFF_W4);
    if ((rc = gemm_bf16(t->dY, OUT, t->w4t, OUT, t->dH, HID, B, HID, OUT, false, st, err))) return rc;
    // layer 3
    k_act_grad<<<nb((size_t)B * HID, 256), 256, 0, st>>>(t->dH, t->Z3, B, HID, t->dZ, t->dZT, t->G + OFF_B3);
    if ((rc = gemm_bf16(t->dZT, B, t->H2T, B, t->G + OFF_W3, HID, HID, HID, B, false, st, err))) return rc;
    if ((rc = gemm_bf16(t->dZ, HID, t->w3t, HID, t->dH, HID, B, HID, HID, false, st, err))) return rc;
    // layer 2
    k_act_grad<<<nb((size_t)B * HID, 256), 256, 0, st>>>(t->dH, t->Z2, B, HID, t->dZ, t->dZT, t->G + OFF_B2);
    if ((rc = gemm_bf16(t->dZT, B, t->H1T, B, t->G + OFF_W2, HID, HID, HID, B, false, st, err))) return rc;
    if ((rc = gemm_bf16(t->dZ, HID, t->w2t, HID, t->dH, HID, B, HID, HID, false, st, err))) return rc;
    // layer 1
    k_act_grad<<<nb((size_t)B * HID, 256), 256, 0, st>>>(t->dH, t->Z1, B, HID, t->dZ, t->dZT, t->G + OFF_B1);
    if ((rc = gemm_bf16(t->dZT, B, t->XT, B, t->G + OFF_W1, IN, HID, IN, B, false, st, err))) return rc;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? AVBD_OK : set_error(AVBD_ERR_CUDA, cudaGetErrorString(e));
}

int avbd_mlp_trainer_grad(avbd_mlp_trainer* t, const void* features, const float* targets, float* loss, float* grad) {
    if (!t || !features || !targets) return set_error(AVBD_ERR_INVALID_ARG, "null argument");
    if (int rc = trainer_fwd_bwd(t, (const bf16*)features, targets)) return rc;
    if (loss) cudaMemcpyAsync(loss, t->loss, sizeof(float), cudaMemcpyDeviceToHost, t->st);
    if (grad) cudaMemcpyAsync(grad, t->G, sizeof(float) * NPAR, cudaMemcpyDeviceToHost, t->st);
    if (cudaStreamSynchronize(t->st) != cudaSuccess) return set_error(AVBD_ERR_CUDA, "trainer sync failed");
    return mlp_device_error(&t->w, t->st);
}

int avbd_mlp_trainer_step(avbd_mlp_trainer* t, const void* features, const float* targets, float lr, float* loss) {
    if (!t || !features || !targets) return set_error(AVBD_ERR_INVALID_ARG, "null argument");
    if (int rc = trainer_fwd_bwd(t, (const bf16*)features, targets)) return rc;
    t->t++;
    const float c1 = 1.0f - powf(0.9f, (float)t->t), c2 = 1.0f - powf(0.999f, (float)t->t);
    k_adam<<<nb(NPAR, 256), 256, 0, t->st>>>(t->w.p32, t->G, t->Mo, t->Vo, lr, c1, c2);
    k_pack<<<nb(HID * HID, 256), 256, 0, t->st>>>(t->w.p32, t->w.w1, t->w.w2, t->w.w3, t->w.w4, t->w1t, t->w2t,
                                                  t->w3t, t->w4t, t->w.b);
    if (loss) {
        cudaMemcpyAsync(loss, t->loss, sizeof(float), cudaMemcpyDeviceToHost, t->st);
        if (cudaStreamSynchronize(t->st) != cudaSuccess) return set_error(AVBD_ERR_CUDA, "trainer sync failed");
        return mlp_device_error(&t->w, t->st);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? AVBD_OK : set_error(AVBD_ERR_CUDA, cudaGetErrorString(e));
}

int avbd_mlp_trainer_get_params(avbd_mlp_trainer* t, float* params) {
    if (!t || !params) return set_error(AVBD_ERR_INVALID_ARG, "null argument");
    cudaMemcpyAsync(params, t->w.p32, sizeof(float) * NPAR, cudaMemcpyDeviceToHost, t->st);
    if (cudaStreamSynchronize(t->st) != cudaSuccess) return set_error(AVBD_ERR_CUDA, "trainer sync failed");
    return mlp_device_error(&t->w, t->st);
}

int avbd_mlp_trainer_destroy(avbd_mlp_trainer* t) {
    if (!t) return AVBD_OK;
    if (t->st) cudaStreamSynchronize(t->st);
    for (void* p : t->allocs) cudaFree(p);
    t->w.release();
    if (t->st) cudaStreamDestroy(t->st);
    delete t;
    return AVBD_OK;
}

}  // extern "C"
