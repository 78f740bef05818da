// The learned far-field closure (no counterpart in the reference): per-particle
// features from the order-1 local expansion, the MLP correction on the
// 5th-generation tensor cores (tcgen05.mma, BF16 operands in shared memory,
// FP32 accumulators in tensor memory), the sampled FP64 judge with fallback
// to the uncorrected forces, and the training kernels (forward on the tensor
// cores with mma.sync m16n8k16, backward and Adam in FP32).
//
// Features of particle i in leaf u (half width h, depth d), with the leaf's
// field L and field gradient G after the order-1 downward pass:
//   s = |L| + h |G|_F
//   x = (L / s, G h / s [xx yy zz xy xz yz], (x_i - c_u) / h, d / 10, 0, 0, 0)
// and the correction is dF_i = m_i s kMlpOutScale MLP(x).
//
// Bounds: the MLP is ~2 x 9.9K flop per particle on the BF16 tensor pipe and
// reads ~80 B per particle; the judge is 4096 x N FP64 pair terms.
#include <algorithm>
#include <cfloat>
#include <cuda_bf16.h>

#include "psg_closure.cuh"
#include "psg_common.cuh"
#include "psg_kernels.h"

namespace psg {

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ float bf16_bits_to_float(uint16_t h) {
    return __uint_as_float((uint32_t)h << 16);
}

__device__ __forceinline__ uint16_t float_to_bf16_bits(float f) {
    __nv_bfloat16 b = __float2bfloat16_rn(f);
    return *reinterpret_cast<uint16_t*>(&b);
}

// D += A (16x16, row) . B (16x8, col), BF16 in, FP32 accumulate
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))
__device__ __forceinline__ float gelu(float x) {
    const float u = 0.7978845608028654f * fmaf(0.044715f * x, x * x, x);
    return 0.5f * x * (1.0f + tanhf(u));
}

__device__ __forceinline__ float gelu_grad(float x) {
    const float x2 = x * x;
    const float u = 0.7978845608028654f * fmaf(0.044715f * x, x2, x);
    const float th = tanhf(u);
    return fmaf(0.5f * x * (1.0f - th * th) * 0.7978845608028654f, fmaf(0.134145f, x2, 1.0f),
                0.5f * (1.0f + th));
}

// One warp, 16 rows: C[16 x 8 NT] = A[16 x 16 KC] . W, A as m16n8k16
// A-fragments, W as Wt[out][in] (row stride LD) in shared memory.
template <int KC, int NT, int LD>
__device__ __forceinline__ void warp_layer(const uint32_t (&a)[KC][4], const uint16_t* wt,
                                           float (&c)[NT][4]) {
    const uint32_t lane = lane_id(), g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
        c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.f;
        const uint16_t* row = wt + (nt * 8 + g) * LD + 2 * t;
#pragma unroll
        for (int kc = 0; kc < KC; ++kc) {
            const uint32_t b0 = *reinterpret_cast<const uint32_t*>(row + kc * 16);
            const uint32_t b1 = *reinterpret_cast<const uint32_t*>(row + kc * 16 + 8);
            mma_bf16(c[nt], a[kc], b0, b1);
        }
    }
}

// z = c + b; h = GELU(z) rounded to BF16 and repacked as the next layer's
// A-fragments (k-chunk kc = n-tiles 2kc and 2kc+1).  With STORE, z (FP32) and
// h (BF16 bits) also go to shared memory rows [16][64] for the backward pass.
template <bool STORE>
__device__ __forceinline__ void act_to_frag(float (&c)[8][4], const float* bias,
                                            uint32_t (&a)[4][4], float* zrow, uint16_t* hrow) {
    const uint32_t lane = lane_id(), g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const int col = nt * 8 + 2 * t;
        const float z0 = c[nt][0] + bias[col], z1 = c[nt][1] + bias[col + 1];
        const float z2 = c[nt][2] + bias[col], z3 = c[nt][3] + bias[col + 1];
        const uint32_t lo = pack_bf16x2(gelu(z0), gelu(z1));
        const uint32_t hi = pack_bf16x2(gelu(z2), gelu(z3));
        const int kc = nt >> 1, half = nt & 1;
        a[kc][half ? 2 : 0] = lo;
        a[kc][half ? 3 : 1] = hi;
        if constexpr (STORE) {
            zrow[g * kMlpHid + col] = z0;
            zrow[g * kMlpHid + col + 1] = z1;
            zrow[(g + 8) * kMlpHid + col] = z2;
            zrow[(g + 8) * kMlpHid + col + 1] = z3;
            *reinterpret_cast<uint32_t*>(hrow + g * kMlpHid + col) = lo;
            *reinterpret_cast<uint32_t*>(hrow + (g + 8) * kMlpHid + col) = hi;
        }
    }
}

// input fragments from feat[16][17] (FP32), rounded to BF16
__device__ __forceinline__ void input_frag(const float (*feat)[17], uint32_t (&a)[1][4]) {
    const uint32_t lane = lane_id(), g = lane >> 2, t = lane & 3;
    a[0][0] = pack_bf16x2(feat[g][2 * t], feat[g][2 * t + 1]);
    a[0][1] = pack_bf16x2(feat[g + 8][2 * t], feat[g + 8][2 * t + 1]);
    a[0][2] = pack_bf16x2(feat[g][2 * t + 8], feat[g][2 * t + 9]);
    a[0][3] = pack_bf16x2(feat[g + 8][2 * t + 8], feat[g + 8][2 * t + 9]);
}

// the whole network on 16 rows; y[16][9] receives the 8 outputs
template <bool STORE>
__device__ __forceinline__ void warp_mlp(const MlpPacked& w, const float (*feat)[17],
                                         float (*y)[9], float* z1, float* z2, float* z3,
                                         uint16_t* h1, uint16_t* h2, uint16_t* h3) {
    const uint32_t lane = lane_id(), g = lane >> 2, t = lane & 3;
    uint32_t a0[1][4];
    input_frag(feat, a0);
    float c[8][4];
    uint32_t a[4][4];
    warp_layer<1, 8, kLd1>(a0, w.wt1, c);
    act_to_frag<STORE>(c, w.b1, a, z1, h1);
    warp_layer<4, 8, kLdH>(a, w.wt2, c);
    act_to_frag<STORE>(c, w.b2, a, z2, h2);
    warp_layer<4, 8, kLdH>(a, w.wt3, c);
    act_to_frag<STORE>(c, w.b3, a, z3, h3);
    float o[1][4];
    warp_layer<4, 1, kLdH>(a, w.wt4, o);
    y[g][2 * t] = o[0][0] + w.b4[2 * t];
    y[g][2 * t + 1] = o[0][1] + w.b4[2 * t + 1];
    y[g + 8][2 * t] = o[0][2] + w.b4[2 * t];
    y[g + 8][2 * t + 1] = o[0][3] + w.b4[2 * t + 1];
}

// features of sorted particle i; returns m_i s kMlpOutScale
__device__ __forceinline__ float closure_features(const TreeView& tv,
                                                  const uint32_t* __restrict__ leaf_of,
                                                  const float4* __restrict__ xyzm, size_t i,
                                                  float* x) {
    const uint32_t u = leaf_of[i];
    if (u >= tv.lvl_base[kLevels]) {  // no leaf recorded: no features, no correction
        for (int k = 0; k < 16; ++k) x[k] = 0.f;
        return 0.f;
    }
    const float4 L = tv.lt[u];
    const float4 g0 = tv.lg0[u];
    const float2 g1 = tv.lg1[u];
    const float4 c = tv.geo[u];
    const float4 p = xyzm[i];
    int depth = 0;
#pragma unroll
    for (int d = 1; d <= kMaxDepth; ++d) depth += u >= tv.lvl_base[d] ? 1 : 0;
    const float h = c.w;
    const float gn = sqrtf(g0.x * g0.x + g0.y * g0.y + g0.z * g0.z +
                           2.0f * (g0.w * g0.w + g1.x * g1.x + g1.y * g1.y));
    const float s = sqrtf(L.y * L.y + L.z * L.z + L.w * L.w) + h * gn + 1e-30f;
    const float is = 1.0f / s;
    const float gh = h * is;
    const float ih = 1.0f / h;
    x[0] = L.y * is;
    x[1] = L.z * is;
    x[2] = L.w * is;
    x[3] = g0.x * gh;
    x[4] = g0.y * gh;
    x[5] = g0.z * gh;
    x[6] = g0.w * gh;
    x[7] = g1.x * gh;
    x[8] = g1.y * gh;
    x[9] = (p.x - c.x) * ih;
    x[10] = (p.y - c.y) * ih;
    x[11] = (p.z - c.z) * ih;
    x[12] = 0.1f * (float)depth;
    x[13] = x[14] = x[15] = 0.f;
    return p.w * s * kMlpOutScale;
}

__device__ __forceinline__ void load_packed(MlpPacked& dst, const MlpPacked* src) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(MlpPacked) / 16); i += blockDim.x) d[i] = s[i];
}

// ---- inference on the 5th-generation tensor cores (tcgen05, TMEM) ----------
// CTAs of 128 threads (4 per SM) take tiles of 128 particles; thread t owns
// row t.  Each layer is D[128 x N] = A[128 x K] . Wt^T (K x N) by
// tcgen05.mma (kind::f16: BF16 operands from shared memory, FP32
// accumulator in tensor memory), issued by one thread, its completion
// signalled on an mbarrier; every thread then reads its row of D from
// tensor memory (tcgen05.ld), adds the bias, applies GELU and writes the
// BF16 row as the next layer's A.  Shared-memory operands are in the
// no-swizzle K-major layout: 8-row x 16-byte core matrices, 128 B apart
// along the rows (the descriptor's stride offset) and R/8 x 128 B apart
// along K (its leading offset) for a matrix of R rows.
constexpr int kTcRows = 128;       // the MMA's M, one particle per row
constexpr uint32_t kTcCols = 64;   // tensor-memory columns: one 128 x 64 FP32 accumulator
constexpr long long kTcWaitCycles = 1ll << 31;  // ~1 s: the bound on an MMA's completion
// CTAs per SM: while one waits on its MMA, the others compute features and
// activations (41 KB of shared memory and 64 tensor-memory columns each)
constexpr int kTcBlocksPerSm = 4;

struct __align__(128) TcSmem {
    uint8_t a0[kTcRows * kMlpIn * 2];   // features, 128 x 16
    uint8_t h[kTcRows * kMlpHid * 2];   // hidden activations, 128 x 64
    uint8_t w1[kMlpHid * kMlpIn * 2];   // Wt1: N = 64 rows x K = 16
    uint8_t w2[kMlpHid * kMlpHid * 2];  // Wt2: 64 x 64
    uint8_t w3[kMlpHid * kMlpHid * 2];  // Wt3: 64 x 64
    uint8_t w4[16 * kMlpHid * 2];       // Wt4: N = 16 rows (8 .. 15 zero) x K = 64
    float b1[kMlpHid], b2[kMlpHid], b3[kMlpHid], b4[16];
    uint64_t mbar;
    uint32_t tmem;
};

// byte offset of element (row, k) of a K-major BF16 operand of `rows` rows
__device__ __forceinline__ uint32_t kmaj_off(uint32_t row, uint32_t k, uint32_t rows) {
    return ((k >> 3) * (rows >> 3) + (row >> 3)) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}

// shared-memory matrix descriptor of a K-major operand at shared address
// saddr (no swizzle; leading offset = rows/8 x 128 B between the two 8-wide
// K chunks of one MMA, stride offset = 128 B between 8-row groups; version 1)
__device__ __forceinline__ uint64_t kmaj_desc(uint32_t saddr, uint32_t rows) {
    const uint64_t lbo = (uint64_t)(rows >> 3) * 128u, sbo = 128u;
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((lbo >> 4) << 16) | ((sbo >> 4) << 32) |
           (1ull << 46);
}

// instruction descriptor: BF16 A and B (K-major), FP32 D, M = 128, N = n
__host__ __device__ constexpr uint32_t tc_idesc(uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) |
           ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// one thread: D (+)= A . B over `ksteps` K-steps of 16, then the commit that
// arrives on the mbarrier when they are done
__device__ __forceinline__ void tc_layer(uint32_t tmem, uint32_t a_addr, uint32_t a_rows,
                                         uint32_t b_addr, uint32_t b_rows, uint32_t idesc,
                                         int ksteps, uint32_t mbar) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    for (int s = 0; s < ksteps; ++s) {
        const uint64_t ad = kmaj_desc(a_addr + (uint32_t)s * 2u * (a_rows >> 3) * 128u, a_rows);
        const uint64_t bd = kmaj_desc(b_addr + (uint32_t)s * 2u * (b_rows >> 3) * 128u, b_rows);
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(s));
    }
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
        : "memory");
}

// wait for the mbarrier's phase `ph` to complete, at most kTcWaitCycles
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t ph) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(mbar), "r"(ph)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > kTcWaitCycles) return false;
    }
}

// this thread's row of the accumulator, columns [c0, c0 + 16)
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// GELU with the hardware's approximate tanh (PTX tanh.approx.f32, relative
// error below 2^-10.9): far below the BF16 rounding every activation gets
// next, and a quarter of the closure network's time against tanhf
__device__ __forceinline__ float gelu_hw(float x) {
    const float u = 0.7978845608028654f * fmaf(0.044715f * x, x * x, x);
    float th;
    asm("tanh.approx.f32 %0, %1;" : "=f"(th) : "f"(u));
    return 0.5f * x * (1.0f + th);
}

// z = D[t] + b; GELU(z) rounded to BF16 into row t of the activations
__device__ __forceinline__ void tc_act(TcSmem& sm, uint32_t trow, const float* bias, uint32_t t) {
#pragma unroll
    for (int c0 = 0; c0 < kMlpHid; c0 += 16) {
        float v[16];
        tc_ld16(trow + (uint32_t)c0, v);
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            uint4 q;
            uint32_t* qq = reinterpret_cast<uint32_t*>(&q);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int k = c0 + half * 8 + 2 * j;
                qq[j] = pack_bf16x2(gelu_hw(v[half * 8 + 2 * j] + bias[k]),
                                    gelu_hw(v[half * 8 + 2 * j + 1] + bias[k + 1]));
            }
            *reinterpret_cast<uint4*>(sm.h + kmaj_off(t, (uint32_t)(c0 + half * 8), kTcRows)) = q;
        }
    }
}

__device__ __forceinline__ void tc_sync() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
}

// FEAT: features from the tree (the closure's correction dF = s y); else
// given inputs x[n][16] -> y[n][8] (the checks of the tensor-core path)
template <bool FEAT>
__global__ void __launch_bounds__(kTcRows, kTcBlocksPerSm)
    k_mlp_tc(TreeView tv, const uint32_t* leaf_of, const float4* __restrict__ xyzm,
             const float* __restrict__ xin, size_t n, const MlpPacked* __restrict__ wts,
             float4* __restrict__ dF, float* __restrict__ yout, uint32_t* err) {
    __shared__ TcSmem sm;
    const uint32_t t = threadIdx.x, w = t >> 5;
    const uint32_t mbar = smem_u32(&sm.mbar);
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (w == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&sm.tmem)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // weights (transposed, BF16) and biases into the operand layout
    for (uint32_t e = t; e < (uint32_t)(kMlpHid * kMlpIn); e += kTcRows) {
        const uint32_t r = e / kMlpIn, k = e % kMlpIn;
        *reinterpret_cast<uint16_t*>(sm.w1 + kmaj_off(r, k, kMlpHid)) = wts->wt1[r * kLd1 + k];
    }
    for (uint32_t e = t; e < (uint32_t)(kMlpHid * kMlpHid); e += kTcRows) {
        const uint32_t r = e / kMlpHid, k = e % kMlpHid;
        *reinterpret_cast<uint16_t*>(sm.w2 + kmaj_off(r, k, kMlpHid)) = wts->wt2[r * kLdH + k];
        *reinterpret_cast<uint16_t*>(sm.w3 + kmaj_off(r, k, kMlpHid)) = wts->wt3[r * kLdH + k];
    }
    for (uint32_t e = t; e < 16u * kMlpHid; e += kTcRows) {
        const uint32_t r = e / kMlpHid, k = e % kMlpHid;
        *reinterpret_cast<uint16_t*>(sm.w4 + kmaj_off(r, k, 16)) =
            r < (uint32_t)kMlpOut ? wts->wt4[r * kLdH + k] : (uint16_t)0;
    }
    if (t < (uint32_t)kMlpHid) {
        sm.b1[t] = wts->b1[t];
        sm.b2[t] = wts->b2[t];
        sm.b3[t] = wts->b3[t];
    }
    if (t < 16) sm.b4[t] = t < (uint32_t)kMlpOut ? wts->b4[t] : 0.f;
    tc_sync();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem;
    const uint32_t trow = tmem + ((w * 32u) << 16);  // this warp's 32 lanes
    const uint32_t a0 = smem_u32(sm.a0), hh = smem_u32(sm.h);
    const uint32_t w1 = smem_u32(sm.w1), w2 = smem_u32(sm.w2), w3 = smem_u32(sm.w3),
                   w4 = smem_u32(sm.w4);
    uint32_t ph = 0;
    bool ok = true;
    const size_t tiles = (n + kTcRows - 1) / kTcRows;
    for (size_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const size_t i = tile * kTcRows + t;
        float x[16];
        float sc = 0.f;
        if (i < n) {
            if constexpr (FEAT) {
                sc = closure_features(tv, leaf_of, xyzm, i, x);
            } else {
#pragma unroll
                for (int k = 0; k < 16; ++k) x[k] = xin[i * 16 + k];
            }
        } else {
#pragma unroll
            for (int k = 0; k < 16; ++k) x[k] = 0.f;
        }
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            uint4 q;
            q.x = pack_bf16x2(x[8 * c + 0], x[8 * c + 1]);
            q.y = pack_bf16x2(x[8 * c + 2], x[8 * c + 3]);
            q.z = pack_bf16x2(x[8 * c + 4], x[8 * c + 5]);
            q.w = pack_bf16x2(x[8 * c + 6], x[8 * c + 7]);
            *reinterpret_cast<uint4*>(sm.a0 + kmaj_off(t, (uint32_t)(8 * c), kTcRows)) = q;
        }
        // layers 1 .. 3 (64 wide), then the output layer (16 wide, 8 used)
        const uint32_t a_addr[4] = {a0, hh, hh, hh};
        const uint32_t b_addr[4] = {w1, w2, w3, w4};
        const float* bias[3] = {sm.b1, sm.b2, sm.b3};
        for (int l = 0; l < 4 && ok; ++l) {
            tc_sync();
            if (t == 0)
                tc_layer(tmem, a_addr[l], kTcRows, b_addr[l], l < 3 ? kMlpHid : 16,
                         tc_idesc(l < 3 ? kMlpHid : 16), l == 0 ? 1 : 4, mbar);
            const bool done = tc_wait(mbar, ph);
            ph ^= 1u;
            ok = !__syncthreads_or(!done);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (l < 3) {
                tc_act(sm, trow, bias[l], t);
            } else {
                float y[16];
                tc_ld16(trow, y);
                if (i < n) {
                    if constexpr (FEAT) {
                        dF[i] = make_float4(sc * (y[0] + sm.b4[0]), sc * (y[1] + sm.b4[1]),
                                            sc * (y[2] + sm.b4[2]), 0.f);
                    } else {
#pragma unroll
                        for (int o = 0; o < kMlpOut; ++o) yout[i * kMlpOut + o] = y[o] + sm.b4[o];
                    }
                }
            }
        }
    }
    if (!ok) {
        // an MMA that did not complete in time: report it, give the last
        // commit one more bounded wait, then release the tensor memory
        if (t == 0) atomicOr(err, PSG_ERR_TC_TIMEOUT);
        tc_wait(mbar, ph ^ 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (w == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTcCols)
                     : "memory");
}

// features (and scale) of selected particles, for building training data
__global__ void __launch_bounds__(256) k_closure_features(TreeView tv, const uint32_t* leaf_of,
                                                          const float4* __restrict__ xyzm,
                                                          size_t n, const uint32_t* idx,
                                                          size_t k, float* __restrict__ x_out,
                                                          float* __restrict__ scale_out) {
    const size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    const uint32_t i = idx[j];
    float x[16];
    float sc = 0.f;
    if (i < n) {
        sc = closure_features(tv, leaf_of, xyzm, i, x);
    } else {
        for (int q = 0; q < 16; ++q) x[q] = 0.f;
    }
    for (int q = 0; q < 16; ++q) x_out[j * 16 + q] = x[q];
    scale_out[j] = sc;
}

// ---- judge ----------------------------------------------------------------
__global__ void k_judge_sample(uint32_t* tg, int s, size_t n, uint32_t tick) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= s) return;
    const size_t stride = n / (size_t)s;
    const size_t off = stride > 1 ? ((size_t)tick * 7919u) % stride : 0;
    size_t i = (size_t)k * n / (size_t)s + off;
    tg[k] = (uint32_t)(i < n ? i : n - 1);
}

// medians of the per-sample relative errors with and without the correction;
// the correction is used only when its median is lower
__global__ void __launch_bounds__(1024) k_judge_decide(const uint32_t* tg, int s,
                                                       const double* f64, const float* fx,
                                                       const float* fy, const float* fz,
                                                       const float4* dF, int allow,
                                                       JudgeOut* out) {
    __shared__ float e0[kJudgeSamples], e1[kJudgeSamples];
    // the sort runs over the smallest power of two >= s, padded with FLT_MAX
    int s2 = 2;
    while (s2 < s && s2 < kJudgeSamples) s2 <<= 1;
    for (int k = threadIdx.x; k < s2; k += blockDim.x) {
        float a = FLT_MAX, b = FLT_MAX;
        if (k < s) {
            const uint32_t i = tg[k];
            const double rx = f64[3 * k], ry = f64[3 * k + 1], rz = f64[3 * k + 2];
            const double nr = sqrt(rx * rx + ry * ry + rz * rz);
            const double bx = (double)fx[i] - rx, by = (double)fy[i] - ry, bz = (double)fz[i] - rz;
            const float4 d = dF[i];
            const double cx = bx + d.x, cy = by + d.y, cz = bz + d.z;
            const double den = nr > 1e-300 ? nr : 1e-300;
            a = (float)(sqrt(bx * bx + by * by + bz * bz) / den);
            b = (float)(sqrt(cx * cx + cy * cy + cz * cz) / den);
        }
        e0[k] = a;
        e1[k] = b;
    }
    __syncthreads();
    // bitonic sort, ascending, both arrays
    for (int size = 2; size <= s2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < s2; i += blockDim.x) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    float x = e0[i], y = e0[j];
                    if ((x > y) == up) {
                        e0[i] = y;
                        e0[j] = x;
                    }
                    x = e1[i];
                    y = e1[j];
                    if ((x > y) == up) {
                        e1[i] = y;
                        e1[j] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        double m0 = 0.0, m1 = 0.0;
        if (s > 0) {
            if (s & 1) {
                m0 = e0[s / 2];
                m1 = e1[s / 2];
            } else {
                m0 = 0.5 * ((double)e0[s / 2 - 1] + (double)e0[s / 2]);
                m1 = 0.5 * ((double)e1[s / 2 - 1] + (double)e1[s / 2]);
            }
        }
        out->median_base = m0;
        out->median_mlp = m1;
        out->use_mlp = (allow && s > 0 && m1 < m0) ? 1 : 0;
        out->samples = s;
    }
}

__global__ void __launch_bounds__(256) k_closure_apply(float* fx, float* fy, float* fz,
                                                       const float4* __restrict__ dF, size_t n,
                                                       const JudgeOut* j) {
    if (!j->use_mlp) return;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float4 d = dF[i];
        fx[i] += d.x;
        fy[i] += d.y;
        fz[i] += d.z;
    }
}

// ---- parameters -------------------------------------------------------------
// FP32 parameter vector -> BF16 transposed weights + FP32 biases
__global__ void k_mlp_pack(const float* __restrict__ p, MlpPacked* __restrict__ out) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    for (int e = tid; e < kMlpHid * kLd1; e += stride) {
        const int o = e / kLd1, i = e % kLd1;
        out->wt1[e] = float_to_bf16_bits(i < kMlpIn ? p[kOffW1 + i * kMlpHid + o] : 0.f);
    }
    for (int e = tid; e < kMlpHid * kLdH; e += stride) {
        const int o = e / kLdH, i = e % kLdH;
        out->wt2[e] = float_to_bf16_bits(i < kMlpHid ? p[kOffW2 + i * kMlpHid + o] : 0.f);
        out->wt3[e] = float_to_bf16_bits(i < kMlpHid ? p[kOffW3 + i * kMlpHid + o] : 0.f);
    }
    for (int e = tid; e < kMlpOut * kLdH; e += stride) {
        const int o = e / kLdH, i = e % kLdH;
        out->wt4[e] = float_to_bf16_bits(i < kMlpHid ? p[kOffW4 + i * kMlpOut + o] : 0.f);
    }
    for (int e = tid; e < kMlpHid; e += stride) {
        out->b1[e] = p[kOffB1 + e];
        out->b2[e] = p[kOffB2 + e];
        out->b3[e] = p[kOffB3 + e];
    }
    for (int e = tid; e < kMlpOut; e += stride) out->b4[e] = p[kOffB4 + e];
}

// ---- training ---------------------------------------------------------------
constexpr int kTrainRows = 64;  // samples per block (4 warps x 16)

struct TrainSmem {
    MlpPacked w;
    uint16_t h0[kTrainRows * kMlpIn];   // BF16 inputs
    uint16_t h1[kTrainRows * kMlpHid];  // BF16 activations
    uint16_t h2[kTrainRows * kMlpHid];
    uint16_t h3[kTrainRows * kMlpHid];
    float z1[kTrainRows * kMlpHid];     // FP32 pre-activations
    float z2[kTrainRows * kMlpHid];
    float z3[kTrainRows * kMlpHid];
    float da[kTrainRows * kMlpHid];     // gradients, ping-pong
    float db[kTrainRows * kMlpHid];
    float dy[kTrainRows * kMlpOut];
    float feat[4][16][17];
    float y[4][16][9];
};

size_t mlp_train_smem_bytes() { return sizeof(TrainSmem); }

// dW[k][n] += sum_b h[b][k] d[b][n]  and  db[n] += sum_b d[b][n]
__device__ __forceinline__ void accum_dw(const uint16_t* h, int K, const float* d, int N,
                                         float* gW, float* gB) {
    for (int e = threadIdx.x; e < K * N; e += blockDim.x) {
        const int n = e / K, k = e % K;
        float sum = 0.f;
        for (int b = 0; b < kTrainRows; ++b) sum = fmaf(bf16_bits_to_float(h[b * K + k]), d[b * N + n], sum);
        atomicAdd(&gW[k * N + n], sum);
    }
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
        float sum = 0.f;
        for (int b = 0; b < kTrainRows; ++b) sum += d[b * N + e];
        atomicAdd(&gB[e], sum);
    }
}

// dnext[b][k] = (sum_n d[b][n] W[k][n]) * GELU'(z[b][k]), W[k][n] = Wt[n][k]
__device__ __forceinline__ void back_act(const float* d, int N, const uint16_t* wt, int ld,
                                         const float* z, float* dnext) {
    for (int e = threadIdx.x; e < kTrainRows * kMlpHid; e += blockDim.x) {
        const int b = e / kMlpHid, k = e % kMlpHid;
        float sum = 0.f;
        for (int n = 0; n < N; ++n) sum = fmaf(d[b * N + n], bf16_bits_to_float(wt[n * ld + k]), sum);
        dnext[e] = sum * gelu_grad(z[e]);
    }
}

// Loss sum_{samples, outputs 0..2} (y - t)^2 and its gradient, scaled by
// inv_norm, accumulated into grad (FP32 parameter layout) and loss_sum.
__global__ void __launch_bounds__(128) k_mlp_grad(const float* __restrict__ X,
                                                  const float* __restrict__ T,
                                                  const uint32_t* __restrict__ perm, size_t b0,
                                                  size_t count, const MlpPacked* __restrict__ wts,
                                                  float inv_norm, float* __restrict__ grad,
                                                  float* __restrict__ loss_sum) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
    load_packed(S.w, wts);
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    const size_t r_blk = (size_t)blockIdx.x * kTrainRows;
    // inputs of this warp's 16 rows
    if (lane < 16) {
        const size_t r = r_blk + w * 16 + lane;
        const bool valid = r < count;
        const size_t src = valid ? (perm ? perm[b0 + r] : b0 + r) : 0;
        for (int k = 0; k < kMlpIn; ++k) {
            const float v = valid ? X[src * kMlpIn + k] : 0.f;
            S.feat[w][lane][k] = v;
            S.h0[(w * 16 + lane) * kMlpIn + k] = float_to_bf16_bits(v);
        }
    }
    __syncthreads();
    const int row0 = w * 16;
    warp_mlp<true>(S.w, S.feat[w], S.y[w], S.z1 + row0 * kMlpHid, S.z2 + row0 * kMlpHid,
                   S.z3 + row0 * kMlpHid, S.h1 + row0 * kMlpHid, S.h2 + row0 * kMlpHid,
                   S.h3 + row0 * kMlpHid);
    __syncwarp();
    float lsum = 0.f;
    if (lane < 16) {
        const size_t r = r_blk + row0 + lane;
        const bool valid = r < count;
        const size_t src = valid ? (perm ? perm[b0 + r] : b0 + r) : 0;
        for (int o = 0; o < kMlpOut; ++o) {
            float d = 0.f;
            if (valid && o < kMlpOutUsed) {
                const float e = S.y[w][lane][o] - T[src * kMlpOutUsed + o];
                lsum = fmaf(e, e, lsum);
                d = 2.0f * e * inv_norm;
            }
            S.dy[(row0 + lane) * kMlpOut + o] = d;
        }
    }
    lsum = warp_sum(lsum);
    if (lane == 0 && lsum != 0.f) atomicAdd(loss_sum, lsum);
    __syncthreads();
    // layer 4
    accum_dw(S.h3, kMlpHid, S.dy, kMlpOut, grad + kOffW4, grad + kOffB4);
    back_act(S.dy, kMlpOut, S.w.wt4, kLdH, S.z3, S.da);
    __syncthreads();
    // layer 3
    accum_dw(S.h2, kMlpHid, S.da, kMlpHid, grad + kOffW3, grad + kOffB3);
    back_act(S.da, kMlpHid, S.w.wt3, kLdH, S.z2, S.db);
    __syncthreads();
    // layer 2
    accum_dw(S.h1, kMlpHid, S.db, kMlpHid, grad + kOffW2, grad + kOffB2);
    back_act(S.db, kMlpHid, S.w.wt2, kLdH, S.z1, S.da);
    __syncthreads();
    // layer 1
    accum_dw(S.h0, kMlpIn, S.da, kMlpHid, grad + kOffW1, grad + kOffB1);
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters
__global__ void k_mlp_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ g, int n, float lr, float beta1, float beta2,
                           float eps, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = fmaf(beta1, m[i], (1.0f - beta1) * gi);
    const float vi = fmaf(beta2, v[i], (1.0f - beta2) * gi * gi);
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// ---- launchers ------------------------------------------------------------------
void launch_closure_mlp(const TreeView& tv, const uint32_t* leaf_of, const float4* xyzm, size_t n,
                        const MlpPacked* w, float4* dF, int sms, uint32_t* err, cudaStream_t st) {
    const size_t tiles = (n + kTcRows - 1) / kTcRows;
    const size_t grid =
        std::max<size_t>(1, std::min<size_t>(tiles, (size_t)sms * kTcBlocksPerSm));
    k_mlp_tc<true><<<(unsigned)grid, kTcRows, 0, st>>>(tv, leaf_of, xyzm, nullptr, n, w, dF,
                                                       nullptr, err);
}

void launch_mlp_forward(const float* x, size_t n, const MlpPacked* w, float* y, int sms,
                        uint32_t* err, cudaStream_t st) {
    const size_t tiles = (n + kTcRows - 1) / kTcRows;
    const size_t grid =
        std::max<size_t>(1, std::min<size_t>(tiles, (size_t)sms * kTcBlocksPerSm));
    k_mlp_tc<false><<<(unsigned)grid, kTcRows, 0, st>>>(TreeView{}, nullptr, nullptr, x, n, w,
                                                        nullptr, y, err);
}

void launch_closure_features(const TreeView& tv, const uint32_t* leaf_of, const float4* xyzm,
                             size_t n, const uint32_t* idx, size_t k, float* x_out,
                             float* scale_out, cudaStream_t st) {
    if (k == 0) return;
    k_closure_features<<<(unsigned)((k + 255) / 256), 256, 0, st>>>(tv, leaf_of, xyzm, n, idx, k,
                                                                    x_out, scale_out);
}

void launch_judge_direct(const float4* xyzm, size_t n, uint32_t* tg, int s, double* f64,
                         uint32_t tick, int blocks, cudaStream_t st, double* part,
                         size_t part_doubles) {
    k_judge_sample<<<(s + 255) / 256, 256, 0, st>>>(tg, s, n, tick);
    launch_direct_f64(xyzm, n, tg, (size_t)s, f64, blocks, st, part, part_doubles);
}

void launch_judge_decide(const uint32_t* tg, int s, const double* f64, const float* fx,
                         const float* fy, const float* fz, const float4* dF, int allow,
                         JudgeOut* out, cudaStream_t st) {
    k_judge_decide<<<1, 1024, 0, st>>>(tg, s, f64, fx, fy, fz, dF, allow, out);
}

void launch_closure_apply(float* fx, float* fy, float* fz, const float4* dF, size_t n,
                          const JudgeOut* j, int sms, cudaStream_t st) {
    size_t grid = (n + 255) / 256;
    const size_t cap = (size_t)sms * 8;
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
    k_closure_apply<<<(unsigned)grid, 256, 0, st>>>(fx, fy, fz, dF, n, j);
}

void launch_mlp_pack(const float* params, MlpPacked* out, cudaStream_t st) {
    k_mlp_pack<<<16, 256, 0, st>>>(params, out);
}

cudaError_t prepare_mlp_grad_kernel() {
    return cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(TrainSmem));
}

void launch_mlp_grad(const float* X, const float* T, const uint32_t* perm, size_t b0,
                     size_t count, const MlpPacked* w, float inv_norm, float* grad,
                     float* loss_sum, cudaStream_t st) {
    if (count == 0) return;
    const unsigned grid = (unsigned)((count + kTrainRows - 1) / kTrainRows);
    k_mlp_grad<<<grid, 128, sizeof(TrainSmem), st>>>(X, T, perm, b0, count, w, inv_norm, grad,
                                                     loss_sum);
}

void launch_mlp_adam(float* p, float* m, float* v, const float* g, int n, float lr, float beta1,
                     float beta2, float eps, float bc1, float bc2, cudaStream_t st) {
    k_mlp_adam<<<(n + 255) / 256, 256, 0, st>>>(p, m, v, g, n, lr, beta1, beta2, eps, bc1, bc2);
}

}  // namespace psg
