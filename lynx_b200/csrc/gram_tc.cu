// Rayleigh-Ritz Gram products on the 5th-generation tensor cores (sm_100a):
//   Ms = dV * Y^T Y,   Hs = dV * Y^T (HY)                  (N x N, FP64 result)
// for FP32 blocks Y, HY of K = Nd grid points x N states (src/solvers/EigenSolver.cpp:622-660,
// the overlap and projected-Hamiltonian products of the Rayleigh-Ritz step).
//
// Precision (integer split, "Ozaki" scheme): the K range is cut into split chunks; in each
// chunk every state column j is rounded to a 23-bit integer on its own power-of-two scale,
//     T = rint(y 2^(22-e)),  e = the exponent of the column's largest |y| (so |T| <= 2^22),
// and T is written as three balanced base-256 digits, T = d1 2^16 + d2 2^8 + d3 with
// d2, d3 in [-128, 127] and |d1| <= 64: three signed int8 slices whose digits have zero mean.
// The slice products with a+b <= 5 (8 of the 9) are formed by tcgen05.mma kind::i8 into four
// int32 accumulators in tensor memory (weights 2^-12, 2^-20, 2^-28, 2^-36 relative to
// 2^(e_i+e_j)), which is exact: no rounding happens in the tensor cores.  The epilogue
// combines the four levels in FP64 and applies 2^(e_i+e_j); the split partials are summed in
// FP64.  The approximations are the rounding of T (half a unit in 2^22 of the column's
// largest element, unbiased) and the one dropped product d3 d3' 2^-44, both far below the
// FP32 rounding of Y itself once summed over K (the result is as accurate as an FP64 product
// of the FP32 data to about 1e-8 of sqrt(Ms_ii Ms_jj)).  An earlier form with three 7-bit
// slices and six products was measured at 2e-7 (Hs) and 1.4e-5 (rotation, relative to the
// column maximum); FP32-accumulating bf16 products carry an accumulation bias that grows with
// K, ~1e-4 relative at 7e5 points.
//
// Kernel structure (one CTA = one 128 x 128 output tile x one K chunk, 4 warps):
//   warp 0 lane 0  : TMA producer, 2-stage ring of the 6 slice tiles (A s1..s3, B s1..s3),
//                    128 rows x 128 int8 each, in the 128-byte-swizzled K-major layout;
//   warp 1 lane 0  : MMA issuer, 32 MMAs per stage (4 K32 sub-steps x 8 slice products),
//                    then tcgen05.commit to release the stage;
//   all 4 warps    : epilogue, tcgen05.ld of the four 128 x 128 int32 accumulators (warp w
//                    owns TMEM lanes 32w..32w+31) and a store of the FP64 partial tile.
// Ms needs only its upper triangle (the Cholesky reads it), so only tiles tm <= tn run.
// Every mbarrier wait is bounded; a timeout sets the error flag, and tensor memory is
// always released before the CTA exits.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <cstring>

#include "kernels.h"
#include "lynx_common.cuh"
#include "stencil_pipe.cuh"

namespace lynxb {
namespace {

constexpr int BM = 128, BN = 128, BK = 128, STAGES = 2;  // BK: int8 K elements (= bytes) per stage row
constexpr int NSLICE = 3;
constexpr int TILE_BYTES = BM * BK;                      // 16 KB, one slice tile
constexpr int STAGE_BYTES = 2 * NSLICE * TILE_BYTES;     // A and B slices: 96 KB
constexpr int TMEM_COLS = 512;                           // 4 accumulators x 128 columns
// Rotation: the epilogue splits each TMEM lane quarter's 128 columns into kRotParts parts, one
// warp each (kRotParts * 4 warps; BN / kRotParts a multiple of 16).
constexpr int kRotParts = 4, kRotThreads = 128 * kRotParts;
// One K element adds at most 64*128 + 128*128 + 128*64 = 2^15 to an accumulator level (|d1| <= 64,
// |d2|, |d3| <= 128), so a K chunk of 511 steps x 128 rows keeps every int32 level below 2^31.
constexpr int kMaxChunkSteps = 511;
// kind::i8 instruction descriptor: D = S32 (bits 4-5 = 2), A = B = signed 8-bit (bits 7-9,
// 10-12 = 1), K-major A and B, N>>3 at bits 17-22, M>>4 at bits 24-28.
constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

// Shared-memory matrix descriptor for a K-major tile of 128-byte rows, 128-byte swizzle:
// 8-row core groups 1024 bytes apart (stride byte offset), descriptor version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;              // leading byte offset (unused by swizzled K-major)
    d |= (uint64_t)(1024u >> 4) << 32;    // stride byte offset
    d |= (uint64_t)1u << 46;              // version
    d |= (uint64_t)2u << 61;              // SWIZZLE_128B
    return d;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(IDESC), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// Exact powers of two, built from the IEEE-754 exponent field (the argument is clamped to the
// normal range; data whose scale leaves it would lose its slices to underflow, not fault).
__device__ __forceinline__ float pow2f(int k) {
    k = max(-126, min(127, k));
    return __int_as_float((127 + k) << 23);
}
__device__ __forceinline__ double pow2d(int k) {
    k = max(-1022, min(1023, k));
    return __longlong_as_double((long long)(1023 + k) << 52);
}

struct GramArgs {
    int ksteps;     // K steps of BK over the whole (padded) K range
    int kper;       // K steps per split
    int nsplit;
    int T;          // tiles along N
    int ntri;       // T (T + 1) / 2: upper-triangular tile pairs of Ms
    int npad;       // T * 128
    const int* eY;  // [nsplit][npad] column exponents of Y
    const int* eH;  // [nsplit][npad] column exponents of HY
    double* ws;     // [2][nsplit][npad][npad] FP64 partial tiles
    int* err;
};

__global__ void __launch_bounds__(128, 1)
    gram_i8_kernel(const __grid_constant__ CUtensorMap tY1, const __grid_constant__ CUtensorMap tY2,
                   const __grid_constant__ CUtensorMap tY3, const __grid_constant__ CUtensorMap tH1,
                   const __grid_constant__ CUtensorMap tH2, const __grid_constant__ CUtensorMap tH3,
                   const GramArgs g) {
    extern __shared__ __align__(1024) unsigned char gsm[];
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(gsm) + 1023) & ~static_cast<uintptr_t>(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(base + STAGES * STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* done = empty + STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int prod, tm, tn;
    if ((int)blockIdx.x < g.ntri) {  // Ms: tile pairs tm <= tn, row by row
        prod = 0;
        int r = blockIdx.x;
        tm = 0;
        while (r >= g.T - tm) {
            r -= g.T - tm;
            ++tm;
        }
        tn = tm + r;
    } else {
        prod = 1;
        const int r = blockIdx.x - g.ntri;
        tm = r / g.T;
        tn = r % g.T;
    }
    const int m0 = tm * BM, n0 = tn * BN;
    const int split = blockIdx.y;
    const int k0 = split * g.kper;
    const int nk = min(g.ksteps, k0 + g.kper) - k0;
    const CUtensorMap* mA[NSLICE] = {&tY1, &tY2, &tY3};
    const CUtensorMap* mB[NSLICE] = {prod ? &tH1 : &tY1, prod ? &tH2 : &tY2, prod ? &tH3 : &tY3};
    auto tileA = [&](int s, int q) { return base + s * STAGE_BYTES + q * TILE_BYTES; };
    auto tileB = [&](int s, int q) { return base + s * STAGE_BYTES + (NSLICE + q) * TILE_BYTES; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const int row = m0 + warp * 32 + lane;
    double* wrow = g.ws + (((long long)prod * g.nsplit + split) * g.npad + row) * g.npad + n0;
    bool ok = true;
    if (nk > 0) {
        if (warp == 0 && lane == 0) {
            for (int k = 0; k < nk; ++k) {
                const int s = k % STAGES, u = k / STAGES;
                if (u > 0 && !mbar_wait(&empty[s], (uint32_t)((u - 1) & 1))) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(&full[s], STAGE_BYTES);
                const int x = (k0 + k) * BK;
#pragma unroll
                for (int q = 0; q < NSLICE; ++q) {
                    tma_load_2d(tileA(s, q), mA[q], x, m0, &full[s]);
                    tma_load_2d(tileB(s, q), mB[q], x, n0, &full[s]);
                }
            }
        } else if (warp == 1 && lane == 0) {
            for (int k = 0; k < nk; ++k) {
                const int s = k % STAGES, u = k / STAGES;
                if (!mbar_wait(&full[s], (uint32_t)(u & 1))) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                uint64_t a[NSLICE], b[NSLICE];
#pragma unroll
                for (int q = 0; q < NSLICE; ++q) {
                    a[q] = sw128_desc(smem_u32(tileA(s, q)));
                    b[q] = sw128_desc(smem_u32(tileB(s, q)));
                }
#pragma unroll
                for (int kk = 0; kk < BK / 32; ++kk) {
                    const uint64_t off = (uint64_t)(kk * 32) >> 4;  // K32 sub-step = 32 bytes along the row
                    const uint32_t acc = (k > 0 || kk > 0) ? 1u : 0u;
                    mma_i8(tmem + 0, a[0] + off, b[0] + off, acc);        // weight 2^-12
                    mma_i8(tmem + 128, a[0] + off, b[1] + off, acc);      // weight 2^-20
                    mma_i8(tmem + 128, a[1] + off, b[0] + off, 1u);
                    mma_i8(tmem + 256, a[0] + off, b[2] + off, acc);      // weight 2^-28
                    mma_i8(tmem + 256, a[1] + off, b[1] + off, 1u);
                    mma_i8(tmem + 256, a[2] + off, b[0] + off, 1u);
                    mma_i8(tmem + 384, a[1] + off, b[2] + off, acc);      // weight 2^-36
                    mma_i8(tmem + 384, a[2] + off, b[1] + off, 1u);
                }
                mma_commit(&empty[s]);
            }
            mma_commit(done);
        }
        __syncwarp();
        if (!mbar_wait(done, 0)) ok = false;
        // tcgen05.ld is warp-collective (.sync.aligned): the decision must be warp-uniform
        ok = __all_sync(0xffffffffu, ok);
        tc_fence_after();
        if (ok) {
            const int* eA = g.eY + (long long)split * g.npad;
            const int* eB = (prod ? g.eH : g.eY) + (long long)split * g.npad;
            const double sa = pow2d(eA[row]);
            const uint32_t lb = (uint32_t)(warp * 32) << 16;
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 16) {
                uint32_t r2[16], r3[16], r4[16], r5[16];
                tmem_ld16(tmem + lb + (uint32_t)c0, r2);
                tmem_ld16(tmem + lb + 128u + (uint32_t)c0, r3);
                tmem_ld16(tmem + lb + 256u + (uint32_t)c0, r4);
                tmem_ld16(tmem + lb + 384u + (uint32_t)c0, r5);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                double v[16];
#pragma unroll
                for (int t = 0; t < 16; ++t) {
                    const double x = (double)(int)r2[t] * 0x1p-12 + (double)(int)r3[t] * 0x1p-20 +
                                     (double)(int)r4[t] * 0x1p-28 + (double)(int)r5[t] * 0x1p-36;
                    v[t] = x * sa * pow2d(eB[n0 + c0 + t]);  // exact: powers of two
                }
                double2* dst = reinterpret_cast<double2*>(wrow + c0);
#pragma unroll
                for (int q = 0; q < 8; ++q) dst[q] = make_double2(v[2 * q], v[2 * q + 1]);
            }
        }
    } else {
        for (int c = 0; c < BN; ++c) wrow[c] = 0.0;  // empty K chunk: the partial tile is zero
    }
    if (!ok && lane == 0) atomicExch(g.err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// T (|T| <= 2^22) -> balanced base-256 digits T = d1 2^16 + d2 2^8 + d3, d2, d3 in [-128, 127],
// |d1| <= 64 (exact integer steps).
__device__ __forceinline__ void digits3(int T, int8_t& a, int8_t& b, int8_t& c) {
    const int d3 = ((T & 0xFF) ^ 0x80) - 0x80;
    const int T1 = (T - d3) >> 8;
    const int d2 = ((T1 & 0xFF) ^ 0x80) - 0x80;
    a = (int8_t)((T1 - d2) >> 8);
    b = (int8_t)d2;
    c = (int8_t)d3;
}
// t = y 2^(22-e), |t| < 2^22 (an exact power-of-two scaling of FP32 y) -> three int8 slices of
// rint(t).
__device__ __forceinline__ void slice3(float t, int8_t& a, int8_t& b, int8_t& c) {
    digits3(__float2int_rn(t), a, b, c);
}

struct SliceArgs {
    int8_t* s[6];     // Y slices 1..3, HY slices 1..3: [n][ldk]
    int* e[2];        // exponents of Y, HY: [nsplit][npad]
    const float* y[2];
    long long ldy, rows, ldk, chunk;
    int npad;
    int* nonfinite;   // set to 1 when an input element is NaN or Inf (may be null)
};

// One K chunk of one column of an FP32 block (blockIdx.z: Y or HY) -> exponent e and three int8
// slices (rows rows..ldk-1 of the padded K range written as zero).  ldy, rows, chunk and ldk
// are multiples of 4, so the chunk is read as float4 and written as char4.
__global__ void __launch_bounds__(256) slice_i8_kernel(const SliceArgs a) {
    __shared__ float red[8];
    const int split = blockIdx.x, j = blockIdx.y, op = blockIdx.z;
    const long long r0 = (long long)split * a.chunk;
    const long long r1 = min(r0 + a.chunk, a.ldk);
    const long long rend = min(r1, a.rows);
    const float* col = a.y[op] + (long long)j * a.ldy;
    float m = 0.0f;
    bool bad = false;  // fmaxf drops NaN, and slicing would turn it into zeros: flag it instead
#pragma unroll 4
    for (long long r = r0 + 4 * threadIdx.x; r < rend; r += 4 * blockDim.x) {
        const float4 v = *reinterpret_cast<const float4*>(col + r);
        m = fmaxf(fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y))), fmaxf(fabsf(v.z), fabsf(v.w)));
        bad |= !(isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w));
    }
    if (bad && a.nonfinite) *a.nonfinite = 1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    m = red[0];
#pragma unroll
    for (int w = 1; w < 8; ++w) m = fmaxf(m, red[w]);
    int E = 0;
    if (m > 0.0f) frexpf(m, &E);  // m = f 2^E, f in [1/2, 1): |y| 2^(22-E) < 2^22
    const int e = (m > 0.0f) ? E : 0;
    if (threadIdx.x == 0) a.e[op][(long long)split * a.npad + j] = e;
    const float sc = pow2f(22 - e);
    int8_t* o1 = a.s[3 * op] + (long long)j * a.ldk;
    int8_t* o2 = a.s[3 * op + 1] + (long long)j * a.ldk;
    int8_t* o3 = a.s[3 * op + 2] + (long long)j * a.ldk;
#pragma unroll 4
    for (long long r = r0 + 4 * threadIdx.x; r < r1; r += 4 * blockDim.x) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (r < a.rows) v = *reinterpret_cast<const float4*>(col + r);
        char4 c1, c2, c3;
        slice3(v.x * sc, reinterpret_cast<int8_t&>(c1.x), reinterpret_cast<int8_t&>(c2.x), reinterpret_cast<int8_t&>(c3.x));
        slice3(v.y * sc, reinterpret_cast<int8_t&>(c1.y), reinterpret_cast<int8_t&>(c2.y), reinterpret_cast<int8_t&>(c3.y));
        slice3(v.z * sc, reinterpret_cast<int8_t&>(c1.z), reinterpret_cast<int8_t&>(c2.z), reinterpret_cast<int8_t&>(c3.z));
        slice3(v.w * sc, reinterpret_cast<int8_t&>(c1.w), reinterpret_cast<int8_t&>(c2.w), reinterpret_cast<int8_t&>(c3.w));
        *reinterpret_cast<char4*>(o1 + r) = c1;
        *reinterpret_cast<char4*>(o2 + r) = c2;
        *reinterpret_cast<char4*>(o3 + r) = c3;
    }
}

// Ms / Hs (column-major N x N, FP64) = dV * sum over splits of the FP64 partial tiles;
// Ms only for tiles on or above the diagonal.
__global__ void gram_reduce_kernel(double* __restrict__ Ms, double* __restrict__ Hs, const double* __restrict__ ws,
                                   int nsplit, int npad, int n, double dV) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;  // column
    const int i = blockIdx.y;                             // row
    const int prod = blockIdx.z;
    if (j >= n) return;
    if (prod == 0 && (i / BM) > (j / BN)) return;
    double s = 0.0;
    const double* p = ws + ((long long)prod * nsplit * npad + i) * npad + j;
    for (int t = 0; t < nsplit; ++t) s += p[(long long)t * npad * npad];
    (prod ? Hs : Ms)[i + (long long)j * n] = dV * s;
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    // looked up once; thread-safe (function-local static initialisation)
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        return nullptr;
    }();
    return fn;
}

// 2-D int8 tensor [rows][ldk] (ldk contiguous), box 128 x 128, 128-byte swizzle.
int make_map(CUtensorMap* m, const int8_t* ptr, long long ldk, int rows) {
    auto enc = get_encode();
    if (!enc) {
        set_error("cuTensorMapEncodeTiled is not available");
        return LYNX_ERR_CUDA;
    }
    cuuint64_t dims[2] = {(cuuint64_t)ldk, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ldk};
    cuuint32_t box[2] = {BK, BM};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(ptr), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// 2-D int8 tensor [rows][ldk] with K extent kext <= ldk (reads past kext are zero-filled).
int make_map_k(CUtensorMap* m, const int8_t* ptr, long long ldk, long long kext, long long rows) {
    auto enc = get_encode();
    if (!enc) {
        set_error("cuTensorMapEncodeTiled is not available");
        return LYNX_ERR_CUDA;
    }
    cuuint64_t dims[2] = {(cuuint64_t)kext, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ldk};
    cuuint32_t box[2] = {BK, BM};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(ptr), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

}  // namespace

GramPlan gram_plan(long long rows, int n) {
    GramPlan p;
    p.ldk = ((rows + BK - 1) / BK) * BK;
    const int ksteps = (int)(p.ldk / BK);
    const int T = (n + BM - 1) / BM;
    p.npad = T * BM;
    const int tiles = T * (T + 1) / 2 + T * T;
    const int need = (ksteps + kMaxChunkSteps - 1) / kMaxChunkSteps;
    int ns = std::max(1, (4 * 148) / tiles);  // about four waves of CTAs over 148 SMs
    ns = std::max(ns, need);
    ns = std::min(ns, ksteps);
    const int kper = (ksteps + ns - 1) / ns;
    p.nsplit = (ksteps + kper - 1) / kper;  // no empty chunks
    p.kper = kper;
    p.slice_bytes = align256((size_t)p.ldk * n);
    p.exp_bytes = align256((size_t)p.nsplit * p.npad * sizeof(int));
    p.ws_bytes = (size_t)2 * p.nsplit * p.npad * p.npad * sizeof(double);
    p.work_bytes = 6 * p.slice_bytes + 2 * p.exp_bytes + p.ws_bytes;
    return p;
}

namespace {

// ---------------------------------------------------------------------------------------------
// Subspace rotation psi = Y W on the tensor cores (src/solvers/EigenSolver.cpp:674-681), same
// exact-slice scheme as the Gram products.  The states of Y are first rescaled by powers of two
// taken from the overlap diagonal (Y~ = Y 2^-d, W~ = 2^d W, so Y~ W~ = Y W and the rows of Y~
// hold numbers of comparable size); each grid-point row of Y~ is then sliced with its own
// exponent e_r over all states, each column of W~ with its own exponent f_j (23-bit integers
// in balanced base-256 digits).  The contraction runs over the states (K = N), so one int32
// accumulation per level covers it exactly, and
//     psi[r][j] = 2^(e_r + f_j) (acc0 2^-12 + acc1 2^-20 + acc2 2^-28 + acc3 2^-36)
// is formed in FP64 and stored straight into the caller's (unpadded) FP64 layout.  Measured
// against FP64 products of the same data, the rotation is as accurate as an FP32 GEMM of the
// same depth (about 1e-6 of each state's largest element).
// ---------------------------------------------------------------------------------------------
struct RotArgs {
    int N;            // states (K extent and output columns)
    int nsteps;       // K stages of BK
    int ntn;          // output column tiles
    long long rows;   // rows of the padded Y block
    int nx, nxp;      // row padding: r = x + nxp * rest, x < nx valid
    const int* erow;     // [rows] row exponents
    const double* fpow;  // [N] column scales 2^f
    double* psi;      // output, column stride ldp, unpadded rows
    long long ldp;
    int* err;
    // optional electron density of the rotated orbitals: dens_w[j] = weight * occupation of
    // state j; this tile's share sum_j dens_w[j] psi[r][j]^2 goes to dens_part[tn * npts + r]
    const double* dens_w;
    double* dens_part;
    long long npts;
};

__global__ void __launch_bounds__(kRotThreads, 1)
    rot_i8_kernel(const __grid_constant__ CUtensorMap tA1, const __grid_constant__ CUtensorMap tA2,
                  const __grid_constant__ CUtensorMap tA3, const __grid_constant__ CUtensorMap tB1,
                  const __grid_constant__ CUtensorMap tB2, const __grid_constant__ CUtensorMap tB3,
                  const RotArgs g) {
    extern __shared__ __align__(1024) unsigned char gsm[];
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(gsm) + 1023) & ~static_cast<uintptr_t>(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(base + STAGES * STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* done = empty + STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tm = blockIdx.x / g.ntn, tn = blockIdx.x % g.ntn;  // column tiles of one row tile adjacent
    const int m0 = tm * BM, n0 = tn * BN;
    const CUtensorMap* mA[NSLICE] = {&tA1, &tA2, &tA3};
    const CUtensorMap* mB[NSLICE] = {&tB1, &tB2, &tB3};
    auto tileA = [&](int s, int q) { return base + s * STAGE_BYTES + q * TILE_BYTES; };
    auto tileB = [&](int s, int q) { return base + s * STAGE_BYTES + (NSLICE + q) * TILE_BYTES; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    bool ok = true;
    if (warp == 0 && lane == 0) {
        for (int k = 0; k < g.nsteps; ++k) {
            const int s = k % STAGES, u = k / STAGES;
            if (u > 0 && !mbar_wait(&empty[s], (uint32_t)((u - 1) & 1))) {
                ok = false;
                break;
            }
            mbar_expect_tx(&full[s], STAGE_BYTES);
            const int x = k * BK;
#pragma unroll
            for (int q = 0; q < NSLICE; ++q) {
                tma_load_2d(tileA(s, q), mA[q], x, m0, &full[s]);
                tma_load_2d(tileB(s, q), mB[q], x, n0, &full[s]);
            }
        }
    } else if (warp == 1 && lane == 0) {
        for (int k = 0; k < g.nsteps; ++k) {
            const int s = k % STAGES, u = k / STAGES;
            if (!mbar_wait(&full[s], (uint32_t)(u & 1))) {
                ok = false;
                break;
            }
            tc_fence_after();
            uint64_t a[NSLICE], b[NSLICE];
#pragma unroll
            for (int q = 0; q < NSLICE; ++q) {
                a[q] = sw128_desc(smem_u32(tileA(s, q)));
                b[q] = sw128_desc(smem_u32(tileB(s, q)));
            }
#pragma unroll
            for (int kk = 0; kk < BK / 32; ++kk) {
                if (k * BK + kk * 32 >= g.N) break;  // K sub-steps past the last state hold zeros only
                const uint64_t off = (uint64_t)(kk * 32) >> 4;
                const uint32_t acc = (k > 0 || kk > 0) ? 1u : 0u;
                mma_i8(tmem + 0, a[0] + off, b[0] + off, acc);
                mma_i8(tmem + 128, a[0] + off, b[1] + off, acc);
                mma_i8(tmem + 128, a[1] + off, b[0] + off, 1u);
                mma_i8(tmem + 256, a[0] + off, b[2] + off, acc);
                mma_i8(tmem + 256, a[1] + off, b[1] + off, 1u);
                mma_i8(tmem + 256, a[2] + off, b[0] + off, 1u);
                mma_i8(tmem + 384, a[1] + off, b[2] + off, acc);
                mma_i8(tmem + 384, a[2] + off, b[1] + off, 1u);
            }
            mma_commit(&empty[s]);
        }
        mma_commit(done);
    }
    __syncwarp();
    if (!mbar_wait(done, 0)) ok = false;
    ok = __all_sync(0xffffffffu, ok);
    tc_fence_after();
    // Epilogue on all warps: warp w reads TMEM lane quarter w % 4 (its 32 rows) and the column
    // part w / 4 of kRotParts, so the stores of several warps per quarter are in flight.
    __shared__ double fps[BN];  // column scales of this tile
    __shared__ double dws[BN];  // density weights of this tile's states
    __shared__ double dpart[kRotParts][BM];
    if (threadIdx.x < BN) {
        fps[threadIdx.x] = (n0 + (int)threadIdx.x < g.N) ? g.fpow[n0 + threadIdx.x] : 0.0;
        dws[threadIdx.x] = (g.dens_w && n0 + (int)threadIdx.x < g.N) ? g.dens_w[n0 + threadIdx.x] : 0.0;
    }
    __syncthreads();
    double dsum = 0.0;  // this thread's row, its part's columns: sum_j w_j psi^2, j in order
    if (ok) {
        const int quarter = warp & 3, part = warp >> 2;
        const long long row = (long long)m0 + quarter * 32 + lane;
        long long ridx = -1;
        double rs = 1.0;
        if (row < g.rows) {
            const long long xr = row % g.nxp, rest = row / g.nxp;
            if (xr < g.nx) ridx = xr + (long long)g.nx * rest;
            rs = pow2d(g.erow[row]);
        }
        const uint32_t lb = (uint32_t)(quarter * 32) << 16;
#pragma unroll 1
        for (int c0 = part * (BN / kRotParts); c0 < (part + 1) * (BN / kRotParts); c0 += 16) {
            uint32_t r2[16], r3[16], r4[16], r5[16];
            tmem_ld16(tmem + lb + (uint32_t)c0, r2);
            tmem_ld16(tmem + lb + 128u + (uint32_t)c0, r3);
            tmem_ld16(tmem + lb + 256u + (uint32_t)c0, r4);
            tmem_ld16(tmem + lb + 384u + (uint32_t)c0, r5);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (ridx >= 0) {
#pragma unroll
                for (int t = 0; t < 16; ++t) {
                    const int j = n0 + c0 + t;
                    if (j < g.N) {
                        const double x = (double)(int)r2[t] * 0x1p-12 + (double)(int)r3[t] * 0x1p-20 +
                                         (double)(int)r4[t] * 0x1p-28 + (double)(int)r5[t] * 0x1p-36;
                        const double v = x * rs * fps[c0 + t];  // exact: powers of two
                        g.psi[(long long)j * g.ldp + ridx] = v;
                        if (g.dens_w) dsum = fma(dws[c0 + t] * v, v, dsum);
                    }
                }
            }
        }
    }
    if (g.dens_w) {
        // the four column parts of each row in order, then one partial per (column tile, row)
        const int quarter = warp & 3, part = warp >> 2;
        dpart[part][quarter * 32 + lane] = dsum;
        __syncthreads();
        if (threadIdx.x < BM) {
            const long long row = (long long)m0 + threadIdx.x;
            if (row < g.rows) {
                const long long xr = row % g.nxp, rest = row / g.nxp;
                if (xr < g.nx) {
                    double t = 0.0;
#pragma unroll
                    for (int q = 0; q < kRotParts; ++q) t += dpart[q][threadIdx.x];
                    g.dens_part[(long long)tn * g.npts + xr + (long long)g.nx * rest] = t;
                }
            }
        }
    }
    if (!ok && lane == 0) atomicExch(g.err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// Column exponents d_i of Y from the overlap diagonal (Ms_ii = dV |y_i|^2): 2^d_i ~ |y_i|.
__global__ void colexp_kernel(const double* __restrict__ Ms, int n, int* __restrict__ d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double v = Ms[i + (long long)i * n];
        d[i] = (v > 0.0) ? ilogb(sqrt(v)) : 0;
    }
}

// Rows of Y 2^-d -> exponent e_r and three int8 digit slices a_q[r][i] (state index contiguous,
// row stride ldk >= N, states N..ldk-1 written as zero).  CTA = 32 consecutive rows, all
// states staged in shared memory [state][row] (row stride 33).
__global__ void __launch_bounds__(256)
    slice_rows_kernel(int8_t* __restrict__ a1, int8_t* __restrict__ a2, int8_t* __restrict__ a3, long long ldk,
                      int* __restrict__ erow, const float* __restrict__ y, long long ldy, long long rows, int N,
                      const int* __restrict__ dcol) {
    extern __shared__ __align__(16) float tsm[];  // [N][33]
    __shared__ int es[32];
    const long long r0 = (long long)blockIdx.x * 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    // eight loads per warp in flight before their stores (one 128-byte row segment each)
    for (int i0 = w; i0 < N; i0 += 64) {
        const long long r = r0 + lane;
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + 8 * u;
            v[u] = (i < N && r < rows) ? y[(long long)i * ldy + r] : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + 8 * u;
            if (i < N) tsm[i * 33 + lane] = v[u] * pow2f(-dcol[i]);
        }
    }
    __syncthreads();
    for (int rr = w; rr < 32; rr += 8) {
        float m = 0.0f;
        for (int i = lane; i < N; i += 32) m = fmaxf(m, fabsf(tsm[i * 33 + rr]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        int E = 0;
        if (m > 0.0f) frexpf(m, &E);
        if (lane == 0) es[rr] = (m > 0.0f) ? E : 0;
    }
    __syncthreads();
    for (int rr = w; rr < 32; rr += 8) {
        const long long r = r0 + rr;
        if (r >= rows) continue;
        const int e = es[rr];
        if (lane == 0) erow[r] = e;
        const float sc = pow2f(22 - e);
        for (int i0 = 4 * lane; i0 < ldk; i0 += 128) {
            char4 o1, o2, o3;
            int8_t* p1 = reinterpret_cast<int8_t*>(&o1);
            int8_t* p2 = reinterpret_cast<int8_t*>(&o2);
            int8_t* p3 = reinterpret_cast<int8_t*>(&o3);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int i = i0 + q;
                slice3((i < N) ? tsm[i * 33 + rr] * sc : 0.0f, p1[q], p2[q], p3[q]);
            }
            *reinterpret_cast<char4*>(a1 + r * ldk + i0) = o1;
            *reinterpret_cast<char4*>(a2 + r * ldk + i0) = o2;
            *reinterpret_cast<char4*>(a3 + r * ldk + i0) = o3;
        }
    }
}

// Columns of 2^d W (FP64, column-major N x N) -> exponent f_j and three int8 digit slices b_q[j][i]
// of rint(2^(d_i + 22 - f_j) W_ij).
__global__ void __launch_bounds__(128)
    slice_w_kernel(int8_t* __restrict__ b1, int8_t* __restrict__ b2, int8_t* __restrict__ b3, long long ldk,
                   double* __restrict__ fpow, const double* __restrict__ W, int N, const int* __restrict__ dcol) {
    __shared__ double red[4];
    const int j = blockIdx.x;
    const double* col = W + (long long)j * N;
    double m = 0.0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) m = fmax(m, fabs(ldexp(col[i], dcol[i])));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    m = fmax(fmax(red[0], red[1]), fmax(red[2], red[3]));
    int E = 0;
    if (m > 0.0) frexp(m, &E);
    const int f = (m > 0.0) ? E : 0;
    if (threadIdx.x == 0) fpow[j] = pow2d(f);
    for (int i = threadIdx.x; i < ldk; i += blockDim.x) {
        const double t = (i < N) ? ldexp(col[i], dcol[i] + 22 - f) : 0.0;  // |t| < 2^22
        int8_t a, b, c;
        digits3(__double2int_rn(t), a, b, c);
        b1[(long long)j * ldk + i] = a;
        b2[(long long)j * ldk + i] = b;
        b3[(long long)j * ldk + i] = c;
    }
}

}  // namespace

int launch_gram_i8(const float* Y, const float* HY, long long ld, long long rows, int n, double dV,
                   const GramPlan& p, void* work, size_t work_bytes, double* Ms, double* Hs, int* err,
                   int* nonfinite, cudaStream_t st) {
    if (work_bytes < p.work_bytes || (reinterpret_cast<uintptr_t>(work) & 255)) {
        set_error("Gram workspace too small or misaligned");
        return LYNX_ERR_BAD_ARG;
    }
    if ((ld % 4) || (rows % 4) || (reinterpret_cast<uintptr_t>(Y) & 15) || (reinterpret_cast<uintptr_t>(HY) & 15)) {
        set_error("tensor-core Gram needs 16-byte aligned columns and a row count divisible by 4");
        return LYNX_ERR_BAD_ARG;
    }
    unsigned char* w = static_cast<unsigned char*>(work);
    int8_t* sl[6];
    for (int q = 0; q < 6; ++q) sl[q] = reinterpret_cast<int8_t*>(w + q * p.slice_bytes);
    int* eY = reinterpret_cast<int*>(w + 6 * p.slice_bytes);
    int* eH = reinterpret_cast<int*>(w + 6 * p.slice_bytes + p.exp_bytes);
    double* ws = reinterpret_cast<double*>(w + 6 * p.slice_bytes + 2 * p.exp_bytes);
    const long long chunk = (long long)p.kper * BK;
    {
        SliceArgs sa;
        for (int q = 0; q < 6; ++q) sa.s[q] = sl[q];
        sa.e[0] = eY;
        sa.e[1] = eH;
        sa.y[0] = Y;
        sa.y[1] = HY;
        sa.ldy = ld;
        sa.rows = rows;
        sa.ldk = p.ldk;
        sa.chunk = chunk;
        sa.npad = p.npad;
        sa.nonfinite = nonfinite;
        dim3 grid(p.nsplit, n, 2);
        slice_i8_kernel<<<grid, 256, 0, st>>>(sa);
        count_launch();
    }
    CUtensorMap m[6];
    for (int q = 0; q < 6; ++q) LYNX_TRY(make_map(&m[q], sl[q], p.ldk, n));
    GramArgs g;
    g.ksteps = (int)(p.ldk / BK);
    g.kper = p.kper;
    g.nsplit = p.nsplit;
    g.T = p.npad / BM;
    g.ntri = g.T * (g.T + 1) / 2;
    g.npad = p.npad;
    g.eY = eY;
    g.eH = eH;
    g.ws = ws;
    g.err = err;
    const size_t smem = STAGES * STAGE_BYTES + 1024 + 256;
    LYNX_CUDA_TRY(smem_cap(gram_i8_kernel, smem));
    dim3 grid(g.ntri + g.T * g.T, p.nsplit);
    gram_i8_kernel<<<grid, 128, smem, st>>>(m[0], m[1], m[2], m[3], m[4], m[5], g);
    {
        dim3 rg((n + 127) / 128, n, 2);
        gram_reduce_kernel<<<rg, 128, 0, st>>>(Ms, Hs, ws, p.nsplit, p.npad, n, dV);
    }
    count_launch(2);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("Gram kernel launch failed: %s", cudaGetErrorString(e));
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

RotPlan rot_plan(long long rows, int n) {
    RotPlan p;
    p.ldk = ((n + 15) / 16) * 16;
    p.a_bytes = align256((size_t)rows * p.ldk);
    p.b_bytes = align256((size_t)n * p.ldk);
    p.erow_bytes = align256((size_t)rows * sizeof(int));
    p.col_bytes = align256((size_t)n * sizeof(double));
    p.work_bytes = 3 * p.a_bytes + 3 * p.b_bytes + p.erow_bytes + 2 * p.col_bytes;
    p.smem_rows = (size_t)n * 33 * sizeof(float);
    return p;
}

bool rot_supported(int n) { return (size_t)n * 33 * sizeof(float) <= 200 * 1024; }

int launch_colexp(const double* Ms, int n, void* work, const RotPlan& p, long long rows, cudaStream_t st) {
    unsigned char* w = static_cast<unsigned char*>(work);
    int* dcol = reinterpret_cast<int*>(w + 3 * p.a_bytes + 3 * p.b_bytes + p.erow_bytes);
    colexp_kernel<<<(n + 127) / 128, 128, 0, st>>>(Ms, n, dcol);
    count_launch();
    return LYNX_OK;
}

// rho[r] (+)= sum over the column tiles t of part[t * npts + r], in tile order.
__global__ void dens_tiles_reduce_kernel(double* __restrict__ rho, const double* __restrict__ part, int ntiles,
                                         long long npts, int accumulate) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < npts;
         r += (long long)gridDim.x * blockDim.x) {
        double s = accumulate ? rho[r] : 0.0;
        for (int t = 0; t < ntiles; ++t) s += part[(long long)t * npts + r];
        rho[r] = s;
    }
}

int launch_rot_i8(const float* Y, long long ldy, long long rows, int nx, int nxp, const double* W, int n,
                  const RotPlan& p, void* work, size_t work_bytes, double* psi, long long ldp, int* err,
                  cudaStream_t st, const RotDensity* dens) {
    if (work_bytes < p.work_bytes || (reinterpret_cast<uintptr_t>(work) & 255) || !rot_supported(n)) {
        set_error("rotation workspace too small or misaligned, or too many states for the tensor-core rotation");
        return LYNX_ERR_BAD_ARG;
    }
    unsigned char* w = static_cast<unsigned char*>(work);
    int8_t* a[3];
    int8_t* b[3];
    for (int q = 0; q < 3; ++q) a[q] = reinterpret_cast<int8_t*>(w + q * p.a_bytes);
    for (int q = 0; q < 3; ++q) b[q] = reinterpret_cast<int8_t*>(w + 3 * p.a_bytes + q * p.b_bytes);
    int* erow = reinterpret_cast<int*>(w + 3 * p.a_bytes + 3 * p.b_bytes);
    int* dcol = reinterpret_cast<int*>(w + 3 * p.a_bytes + 3 * p.b_bytes + p.erow_bytes);
    double* fpow = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(dcol) + p.col_bytes);
    LYNX_CUDA_TRY(smem_cap(slice_rows_kernel, p.smem_rows));
    slice_rows_kernel<<<(unsigned)((rows + 31) / 32), 256, p.smem_rows, st>>>(a[0], a[1], a[2], p.ldk, erow, Y, ldy,
                                                                               rows, n, dcol);
    slice_w_kernel<<<n, 128, 0, st>>>(b[0], b[1], b[2], p.ldk, fpow, W, n, dcol);
    count_launch(2);
    CUtensorMap m[6];
    for (int q = 0; q < 3; ++q) LYNX_TRY(make_map_k(&m[q], a[q], p.ldk, n, rows));
    for (int q = 0; q < 3; ++q) LYNX_TRY(make_map_k(&m[3 + q], b[q], p.ldk, n, n));
    RotArgs g;
    g.N = n;
    g.nsteps = (n + BK - 1) / BK;
    g.ntn = (n + BN - 1) / BN;
    g.rows = rows;
    g.nx = nx;
    g.nxp = nxp;
    g.erow = erow;
    g.fpow = fpow;
    g.psi = psi;
    g.ldp = ldp;
    g.err = err;
    g.dens_w = dens ? dens->w : nullptr;
    g.dens_part = dens ? dens->part : nullptr;
    g.npts = dens ? dens->npts : 0;
    const size_t smem = STAGES * STAGE_BYTES + 1024 + 256;
    LYNX_CUDA_TRY(smem_cap(rot_i8_kernel, smem));
    const long long ntm = (rows + BM - 1) / BM;
    rot_i8_kernel<<<(unsigned)(ntm * g.ntn), kRotThreads, smem, st>>>(m[0], m[1], m[2], m[3], m[4], m[5], g);
    count_launch();
    if (dens) {
        const int blocks = (int)std::min<long long>((dens->npts + 255) / 256, 148LL * 8);
        dens_tiles_reduce_kernel<<<blocks, 256, 0, st>>>(dens->rho, dens->part, g.ntn, dens->npts,
                                                         dens->accumulate ? 1 : 0);
        count_launch();
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("rotation kernel launch failed: %s", cudaGetErrorString(e));
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

}  // namespace lynxb
