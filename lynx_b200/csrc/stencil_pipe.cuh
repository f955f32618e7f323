// Pipelined fused Chebyshev-filter step for sm_100a (the filter's hot kernel):
//   out = a * (-0.5 * Lap x + Veff .* x) + b * x + d * xold
// (src/solvers/EigenSolver.cpp:586-607 recurrence, src/operators/Hamiltonian.cpp:127-174
// stencil, src/parallel/HaloExchange.cpp:34-189 ghost rules: periodic wrap, Bloch phase
// e^{-+ik_dL_d} on left/right ghosts, zero for Dirichlet), with the ghosts produced in
// the kernel: no padded copy of x is ever written to HBM.
//
// Data layout: blocks of ncol columns, each column a z-major stack of planes of ny rows,
// rows padded to nxp >= nx elements (nxp * sizeof(T) a multiple of 16 bytes, pad
// elements zero), column stride ld (a multiple of 16 bytes).
//
// Work decomposition: one CTA = one column x one band of TY rows x one chunk of z-planes,
// marching through z.  Per plane the CTA needs
//   (a) the band's rows plus R halo rows above and below (y-wrapped) for the x/y
//       derivatives -> staged in shared memory by one elected thread with 1-D bulk
//       async copies (cp.async.bulk, one per row) completing on an mbarrier;
//   (b) xold and Veff on the band's rows -> one bulk copy each into the same stage;
//   (c) the z-neighbours of every owned point -> a register window of 2R+1 planes fed
//       by vector global loads issued two planes ahead.
// The shared-memory ring holds P+1 stages, so the copies for plane z+P are in flight
// while plane z is computed: memory-level parallelism comes from the async copies, not
// from resident warps.  x-ghost columns of a staged plane are filled by the threads
// (periodic or Bloch) after its copies land.  Each thread computes an RX x RY block of
// points (RX adjacent x, RY adjacent y) so the x/y neighbour reads are vector
// shared-memory loads reused across the block.
//
// HBM traffic per update: x, xold and out once each (3 words).  Halo rows and Veff are
// re-read from L2.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "stencil.cuh"

namespace lynxb {

constexpr int kPipeStages = 3;        // P + 1
constexpr int kPipeMaxThreads = 384;
constexpr long long kSpinLimit = 1LL << 22;  // bounded mbarrier waits

struct PipeGeom {
    int nx, ny, nz;
    int nxp;           // padded row length (elements)
    int SP;            // staged row pitch (elements)
    int GL;            // left ghost columns in a staged row (>= R, 16-byte multiple)
    int TYT, TY;       // thread rows, band height
    int P2;            // x-blocks per thread row (ceil(nx / RX))
    int zchunk;
    long long plane;   // nxp * ny
    long long ld_x, ld_old, ld_out;
};

template <typename T>
struct PipeCoef {
    using S = typename ScalarOf<T>::type;
    S cx[9], cy[9], cz[9];
    S diag, a, d;
    T phl[3], phr[3];
};

template <typename T, int RX> struct VecOf { using type = T; };
template <> struct VecOf<float, 2> { using type = float2; };
template <> struct VecOf<double, 2> { using type = double2; };

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait for the phase with the given parity; returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    for (long long i = 0; i < kSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Pipelined kernel.  RX adjacent x points and RY adjacent rows per thread.
template <typename T, int R, int RX, int RY, bool XOLD>
__global__ void __launch_bounds__(kPipeMaxThreads)
    cheb_pipe_kernel(const T* __restrict__ x, const T* __restrict__ xold, T* __restrict__ out,
                     const typename ScalarOf<T>::type* __restrict__ V, const PipeGeom G, const PipeCoef<T> C,
                     int* __restrict__ err) {
    using S = typename ScalarOf<T>::type;
    using VT = typename VecOf<T, RX>::type;
    constexpr int W = 2 * R + 1;
    constexpr int NS = kPipeStages;
    constexpr int P = NS - 1;
    // x-neighbour vector loads: first element index rounded down to a multiple of RX
    constexpr int XOFF = (R % RX == 0) ? R : (R + RX - (R % RX));  // XOFF >= R, XOFF % RX == 0
    constexpr int NXV = (XOFF + R + RX + RX - 1) / RX;            // vectors covering x-XOFF .. x+RX-1+R

    extern __shared__ __align__(128) unsigned char smpipe[];
    const int tid = threadIdx.x;
    const int nthr = blockDim.x;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const int y0 = blockIdx.x * G.TY;
    const int TYv = min(G.TY, ny - y0);
    const int z0 = blockIdx.z * G.zchunk;
    const int z1 = min(nz, z0 + G.zchunk);
    const long long col = blockIdx.y;
    const T* __restrict__ xc = x + col * G.ld_x;
    const T* __restrict__ xoc = XOLD ? xold + col * G.ld_old : nullptr;
    T* __restrict__ oc = out + col * G.ld_out;

    // Shared-memory carve-up: [mbarriers][stage 0][stage 1]...; a stage holds the staged
    // tile ((TY + 2R) rows of pitch SP), then xold rows and Veff rows (TY x nxp each).
    const int tile_elems = (G.TY + 2 * R) * G.SP;
    const int own_elems = G.TY * G.nxp;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smpipe);
    T* stage0 = reinterpret_cast<T*>(smpipe + 128);
    const int stage_bytes_T = (tile_elems + (XOLD ? own_elems : 0)) * (int)sizeof(T);
    const int stage_stride = ((stage_bytes_T + own_elems * (int)sizeof(S) + 127) / 128) * 128;
    auto tile_of = [&](int s) { return reinterpret_cast<T*>(reinterpret_cast<unsigned char*>(stage0) + s * stage_stride); };
    auto xold_of = [&](int s) { return tile_of(s) + tile_elems; };
    auto veff_of = [&](int s) {
        return reinterpret_cast<S*>(reinterpret_cast<unsigned char*>(tile_of(s)) + stage_bytes_T);
    };

    if (tid == 0) {
        for (int s = 0; s < NS; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
    }
    __syncthreads();

    // Producer: all copies of plane z into stage s (elected thread 0).
    auto issue = [&](int z, int s) {
        T* tile = tile_of(s);
        const uint32_t rowb = (uint32_t)(G.nxp * sizeof(T));
        const uint32_t ownb = (uint32_t)(TYv * G.nxp * sizeof(T));
        const uint32_t vb = (uint32_t)(TYv * G.nxp * sizeof(S));
        const uint32_t total = (uint32_t)(TYv + 2 * R) * rowb + (XOLD ? ownb : 0u) + vb;
        fence_proxy_async_smem();
        mbar_expect_tx(&bars[s], total);
        const T* plane = xc + (long long)z * G.plane;
        for (int t = 0; t < TYv + 2 * R; ++t) {
            int gy = y0 - R + t;
            gy += (gy < 0) ? ny : 0;
            gy -= (gy >= ny) ? ny : 0;
            bulk_g2s(tile + t * G.SP + G.GL, plane + (long long)gy * G.nxp, rowb, &bars[s]);
        }
        const long long own0 = (long long)z * G.plane + (long long)y0 * G.nxp;
        if (XOLD) bulk_g2s(xold_of(s), xoc + own0, ownb, &bars[s]);
        bulk_g2s(veff_of(s), V + (long long)z * G.plane + (long long)y0 * G.nxp, vb, &bars[s]);
    };

    // Thread block of points.
    const int px = tid % G.P2;
    const int ty = tid / G.P2;
    const int xb = px * RX;  // first x of the block
    int yl[RY];
    bool own[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        yl[r] = ty * RY + r;
        own[r] = (ty < G.TYT) && (yl[r] < TYv);
    }
    const T zero = vzero(T());

    auto load_own_plane = [&](int zz, VT* v) {
        T mul = C.phl[2];
        bool wrapped = false;
        if (zz < 0) {
            zz += nz;
            wrapped = true;
        } else if (zz >= nz) {
            zz -= nz;
            mul = C.phr[2];
            wrapped = true;
        }
        const T* base = xc + (long long)zz * G.plane + (long long)y0 * G.nxp + xb;
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            VT t;
            if (own[r]) {
                t = *reinterpret_cast<const VT*>(base + (long long)yl[r] * G.nxp);
            } else {
                T* tp = reinterpret_cast<T*>(&t);
#pragma unroll
                for (int i = 0; i < RX; ++i) tp[i] = zero;
            }
            if (wrapped) {
                T* tp = reinterpret_cast<T*>(&t);
#pragma unroll
                for (int i = 0; i < RX; ++i) tp[i] = pmul(tp[i], mul);
            }
            v[r] = t;
        }
    };

    // Prologue: copies for the first P planes, window for the first plane, two planes of
    // window prefetch.
    if (tid == 0) {
        for (int i = 0; i < P; ++i)
            if (z0 + i < z1) issue(z0 + i, i);
    }
    VT w[W][RY];
#pragma unroll
    for (int k = 0; k < W; ++k) load_own_plane(z0 - R + k, w[k]);
    VT pf0[RY], pf1[RY];
    load_own_plane(z0 + R + 1, pf0);
    load_own_plane(z0 + R + 2, pf1);

    const T phl_x = C.phl[0], phr_x = C.phr[0];
    const T phl_y = C.phl[1], phr_y = C.phr[1];
    const bool wrap_top = (y0 - R) < 0;
    const bool wrap_bot = (y0 + TYv + R) > ny;
    const int ghost_rows = TYv + 2 * R;

    for (int z = z0; z < z1; ++z) {
        const int it = z - z0;
        const int s = it % NS;
        __syncthreads();  // S1: every thread is done with iteration it-1 (stage (it+P) % NS is free)
        if (tid == 0 && z + P < z1) issue(z + P, (it + P) % NS);
        // Wait for plane z.
        bool ok = mbar_wait(&bars[s], (uint32_t)((it / NS) & 1));
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(err, 1);
            return;
        }
        T* tile = tile_of(s);
        // Bloch phase / Dirichlet zero on y-wrapped halo rows (rows copied from the other side).
        if (ScalarOf<T>::cplx || wrap_top || wrap_bot) {
            if (wrap_top || wrap_bot) {
                for (int e = tid; e < 2 * R * nx; e += nthr) {
                    const int hr = e / nx, hx = e - (e / nx) * nx;
                    const int t = (hr < R) ? hr : (TYv + hr);
                    const int gy = y0 - R + t;
                    if (gy < 0) tile[t * G.SP + G.GL + hx] = pmul(tile[t * G.SP + G.GL + hx], phl_y);
                    else if (gy >= ny) tile[t * G.SP + G.GL + hx] = pmul(tile[t * G.SP + G.GL + hx], phr_y);
                }
                __syncthreads();
            }
        }
        // x-ghost columns: left ghost x' = -p holds x(nx - p) * phl, right ghost x' = nx + p
        // holds x(p) * phr.
        for (int e = tid; e < ghost_rows * 2 * R; e += nthr) {
            const int t = e / (2 * R);
            const int g = e - t * (2 * R);
            T* row = tile + t * G.SP + G.GL;
            if (g < R) row[-R + g] = pmul(row[nx - R + g], phl_x);
            else row[nx + (g - R)] = pmul(row[g - R], phr_x);
        }
        __syncthreads();  // S2: plane z staged with ghosts

        // Compute the RX x RY block of plane z.
        const T* xo_s = XOLD ? xold_of(s) : nullptr;
        const S* v_s = veff_of(s);
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            if (!own[r]) continue;
            const int row = R + yl[r];
            const T* trow = tile + row * G.SP + G.GL + xb;
            T acc[RX];
            const T* wc = reinterpret_cast<const T*>(&w[R][r]);
#pragma unroll
            for (int i = 0; i < RX; ++i) acc[i] = vscale(C.diag, wc[i]);
            // x neighbours: vectors covering x-XOFF .. x+RX-1+R
            {
                T xv[NXV * RX];
#pragma unroll
                for (int k = 0; k < NXV; ++k)
                    *reinterpret_cast<VT*>(&xv[k * RX]) = *reinterpret_cast<const VT*>(trow - XOFF + k * RX);
#pragma unroll
                for (int i = 0; i < RX; ++i)
#pragma unroll
                    for (int p = 1; p <= R; ++p)
                        acc[i] = fmac(acc[i], C.cx[p], vadd(xv[XOFF + i + p], xv[XOFF + i - p]));
            }
            // y neighbours
#pragma unroll
            for (int p = 1; p <= R; ++p) {
                const VT up = *reinterpret_cast<const VT*>(trow + p * G.SP);
                const VT dn = *reinterpret_cast<const VT*>(trow - p * G.SP);
                const T* u = reinterpret_cast<const T*>(&up);
                const T* dd = reinterpret_cast<const T*>(&dn);
#pragma unroll
                for (int i = 0; i < RX; ++i) acc[i] = fmac(acc[i], C.cy[p], vadd(u[i], dd[i]));
            }
            // z neighbours
#pragma unroll
            for (int p = 1; p <= R; ++p) {
                const T* u = reinterpret_cast<const T*>(&w[R + p][r]);
                const T* dd = reinterpret_cast<const T*>(&w[R - p][r]);
#pragma unroll
                for (int i = 0; i < RX; ++i) acc[i] = fmac(acc[i], C.cz[p], vadd(u[i], dd[i]));
            }
            const int so = yl[r] * G.nxp + xb;
#pragma unroll
            for (int i = 0; i < RX; ++i) {
                acc[i] = fmac(acc[i], C.a * v_s[so + i], wc[i]);
                if (XOLD) acc[i] = fmac(acc[i], C.d, xo_s[so + i]);
            }
            T* op = oc + (long long)z * G.plane + (long long)(y0 + yl[r]) * G.nxp + xb;
            if (xb + RX <= nx) {
                VT o;
                T* opv = reinterpret_cast<T*>(&o);
#pragma unroll
                for (int i = 0; i < RX; ++i) opv[i] = acc[i];
                *reinterpret_cast<VT*>(op) = o;
            } else {
#pragma unroll
                for (int i = 0; i < RX; ++i)
                    if (xb + i < nx) op[i] = acc[i];
            }
        }

        // Slide the window and the prefetch.
#pragma unroll
        for (int k = 0; k < W - 1; ++k)
#pragma unroll
            for (int r = 0; r < RY; ++r) w[k][r] = w[k + 1][r];
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            w[W - 1][r] = pf0[r];
            pf0[r] = pf1[r];
        }
        if (z + 1 < z1) load_own_plane(z + R + 3, pf1);
    }
}

}  // namespace lynxb
