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
#include <type_traits>

#include "stencil.cuh"

namespace lynxb {

constexpr int kPipeMaxThreads = 352;
constexpr int kSpinLimit = 1 << 22;  // bounded mbarrier waits (a 32-bit counter: cheaper per wait)

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
    S diag, diag_lo, a, d;  // centre coefficient as a (hi, lo) pair (centre_coef)
    T phl[3], phr[3];
};

// Fused nonlocal term (real data, disjoint projector spheres): W holds (chi alpha) per sphere
// point in grid order (column stride ldw); ptmap (row pitch mp, same rows as the grid) gives
// each grid point's number in that order, or -1; rowstart[z * ny + y] is the number of the
// first sphere point at or after row (z, y).  wcap: the largest W range of one band-plane,
// rounded out to 16-byte boundaries.
template <typename T>
struct PipeNL {
    const T* W;
    long long ldw;
    const int* ptmap;
    int mp;
    const int* rowstart;
    int wcap;
    T* xs_out;  // optional: compact copy of out at the sphere points (column stride ldw)
};

// Byte layout of one tile stage: [tile rows][xold rows][Veff rows][ptmap rows][W range],
// every part 16-byte aligned; returns the 128-byte rounded stage size.
struct StageLayout {
    int v_off, pm_off, w_off, bytes;
};
__host__ __device__ inline StageLayout pipe_stage_layout(int TY, int R, int nxp, int szT, int szS, bool xold, bool nlf,
                                                        int mp, int wcap) {
    StageLayout L;
    const int tb = ((TY + 2 * R) * nxp + (xold ? TY * nxp : 0)) * szT;
    L.v_off = (tb + 15) & ~15;
    L.pm_off = (L.v_off + TY * nxp * szS + 15) & ~15;
    L.w_off = (L.pm_off + (nlf ? TY * mp * 4 : 0) + 15) & ~15;
    L.bytes = ((L.w_off + (nlf ? wcap * szT : 0) + 127) / 128) * 128;
    return L;
}

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

// Bounded wait for the phase with the given parity (at most `limit` tries); returns false on
// timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit = kSpinLimit) {
    const uint32_t addr = smem_u32(bar);
    for (int i = 0; i < limit; ++i) {
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

// Shared-memory loads at 32-bit shared-window addresses.  The consumers keep per-thread byte
// offsets and advance them by additions; written through generic pointers, every neighbour
// address cost 64-bit pointer arithmetic, and the integer work outweighed the floating point.
template <typename V> __device__ __forceinline__ V lds(uint32_t a);
template <> __device__ __forceinline__ float lds<float>(uint32_t a) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
    return v;
}
template <> __device__ __forceinline__ double lds<double>(uint32_t a) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
    return v;
}
template <> __device__ __forceinline__ float2 lds<float2>(uint32_t a) {
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
    return v;
}
template <> __device__ __forceinline__ double2 lds<double2>(uint32_t a) {
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
    return v;
}
template <> __device__ __forceinline__ int2 lds<int2>(uint32_t a) {
    int2 v;
    asm volatile("ld.shared.v2.s32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(a));
    return v;
}
template <> __device__ __forceinline__ int lds<int>(uint32_t a) {
    int v;
    asm volatile("ld.shared.s32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Warp-specialised pipelined kernel.  The last warp of the CTA is the producer: it keeps
// NS stages of the shared-memory ring in flight with bulk copies (the band's rows plus R
// halo rows on each side as one contiguous copy, two where the band meets the y boundary;
// xold and Veff rows; and, in a separate DW-stage ring, the rows of the plane entering the
// z-window).  The other warps are consumers: each thread computes RX adjacent x points on
// RY adjacent rows.  Staged rows carry no ghost columns: a consumer reads its x neighbours
// through column offsets wrapped once at start-up, and PHASED instantiations (Bloch phases,
// Dirichlet zeros) multiply wrapped neighbours in registers.  Per stage two mbarriers:
// full (copies landed, tx-counted) and empty (every consumer warp done reading).
template <typename T, int R, int RX, int RY, bool XOLD, int NS, bool PHASED, int MAXT, bool NLF>
__global__ void __launch_bounds__(MAXT, 1)
    cheb_pipe_kernel(const T* __restrict__ x, const T* __restrict__ xold, T* __restrict__ out,
                     const typename ScalarOf<T>::type* __restrict__ V, const PipeGeom G, const PipeCoef<T> C,
                     const PipeNL<T> NL, int* __restrict__ err) {
    using S = typename ScalarOf<T>::type;
    using VT = typename VecOf<T, RX>::type;
    constexpr int W = 2 * R + 1;
    constexpr int DW = 4;  // window ring depth
    static_assert((2 * NS + 2 * DW) * 8 <= 192 && NS <= 16, "ring size out of range");  // 192..255: W offsets
    // x-neighbour vector loads: first element index rounded down to a multiple of RX
    constexpr int XOFF = (R % RX == 0) ? R : (R + RX - (R % RX));  // XOFF >= R, XOFF % RX == 0
    constexpr int NXV = (XOFF + R + RX + RX - 1) / RX;            // vectors covering x-XOFF .. x+RX-1+R
    constexpr bool kPacked = std::is_same<T, float>::value && RX == 2;

    extern __shared__ __align__(128) unsigned char smpipe[];
    const int tid = threadIdx.x;
    const int NC = blockDim.x - 32;  // consumer threads (a multiple of 32)
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const int nxp = G.nxp;
    const int y0 = blockIdx.x * G.TY;
    const int TYv = min(G.TY, ny - y0);
    const int z0 = blockIdx.z * G.zchunk;
    const int z1 = min(nz, z0 + G.zchunk);
    const int nplanes = z1 - z0;
    const long long col = blockIdx.y;
    const T* __restrict__ xc = x + col * G.ld_x;
    const T* __restrict__ xoc = XOLD ? xold + col * G.ld_old : nullptr;
    T* __restrict__ oc = out + col * G.ld_out;

    // Shared memory: [mbarriers][NS tile stages][DW window stages]; a tile stage holds
    // (TY + 2R) rows of the plane (pitch nxp), then xold and Veff on the band's rows.
    const int tile_elems = (G.TY + 2 * R) * nxp;
    const int own_elems = G.TY * nxp;
    uint64_t* full = reinterpret_cast<uint64_t*>(smpipe);
    uint64_t* empty = full + NS;
    uint64_t* wfull = empty + NS;
    uint64_t* wempty = wfull + DW;
    T* stage0 = reinterpret_cast<T*>(smpipe + 256);
    int* walign = reinterpret_cast<int*>(smpipe + 192);  // per stage: first W element staged
    const StageLayout SL = pipe_stage_layout(G.TY, R, nxp, (int)sizeof(T), (int)sizeof(S), XOLD, NLF, NL.mp, NL.wcap);
    const int stage_stride = SL.bytes;
    const int wstage_stride = ((own_elems * (int)sizeof(T) + 127) / 128) * 128;
    auto tile_of = [&](int st) {
        return reinterpret_cast<T*>(reinterpret_cast<unsigned char*>(stage0) + st * stage_stride);
    };
    auto xold_of = [&](int st) { return tile_of(st) + tile_elems; };
    auto veff_of = [&](int st) {
        return reinterpret_cast<S*>(reinterpret_cast<unsigned char*>(tile_of(st)) + SL.v_off);
    };
    auto pm_of = [&](int st) {
        return reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(tile_of(st)) + SL.pm_off);
    };
    auto wnl_of = [&](int st) {
        return reinterpret_cast<T*>(reinterpret_cast<unsigned char*>(tile_of(st)) + SL.w_off);
    };
    auto wstage_of = [&](int st) {
        return reinterpret_cast<T*>(reinterpret_cast<unsigned char*>(stage0) + NS * stage_stride + st * wstage_stride);
    };

    if (tid == 0) {
        for (int st = 0; st < NS; ++st) {
            mbar_init(&full[st], 1);
            mbar_init(&empty[st], NC / 32);
        }
        for (int st = 0; st < DW; ++st) {
            mbar_init(&wfull[st], 1);
            mbar_init(&wempty[st], NC / 32);
        }
        fence_mbar_init();
    }
    __syncthreads();

    if (tid >= NC) {
        // ------------------------------ producer warp ------------------------------
        // W ranges of this band on every plane of the chunk, read once by the whole warp
        // (after the window ring): rsv[2i], rsv[2i+1] = first / end compact point of plane z0+i.
        int* rsv = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(stage0) + NS * stage_stride +
                                          DW * wstage_stride);
        if constexpr (NLF) {
            for (int i = tid - NC; i < nplanes; i += 32) {
                const long long rb = (long long)(z0 + i) * ny + y0;
                rsv[2 * i] = NL.rowstart[rb];
                rsv[2 * i + 1] = NL.rowstart[rb + TYv];
            }
            __syncwarp();
        }
        if (tid != NC) return;  // one elected thread issues every copy
        const uint32_t rowb = (uint32_t)(nxp * sizeof(T));
        const uint32_t ownb = (uint32_t)(TYv * nxp * sizeof(T));
        const uint32_t vb = (uint32_t)(TYv * nxp * sizeof(S));
        const int nrows = TYv + 2 * R;
        const uint32_t total = (uint32_t)nrows * rowb + (XOLD ? ownb : 0u) + vb;
        // rows y0-R .. y0+TYv+R-1 as up to three contiguous runs of global rows (y wraps)
        int run_t[3], run_y[3], run_n[3], nruns = 0;
        {
            int t = 0;
            while (t < nrows) {
                int gy = y0 - R + t;
                gy += (gy < 0) ? ny : 0;
                gy -= (gy >= ny) ? ny : 0;
                const int n = min(nrows - t, ny - gy);
                run_t[nruns] = t;
                run_y[nruns] = gy;
                run_n[nruns] = n;
                ++nruns;
                t += n;
            }
        }
        for (int i = 0; i < nplanes; ++i) {
            const int z = z0 + i;
            const int st = i % NS, k = i / NS;
            if (k > 0 && !mbar_wait(&empty[st], (uint32_t)((k - 1) & 1))) {
                atomicExch(err, 1);
                return;
            }
            uint32_t extra = 0, pmb = 0, wnb = 0;
            int wal = 0;
            if constexpr (NLF) {
                constexpr int VWn = 16 / (int)sizeof(T);
                const int ps = rsv[2 * i], pe = rsv[2 * i + 1];
                wal = ps & ~(VWn - 1);
                const int wae = (pe + VWn - 1) & ~(VWn - 1);
                walign[st] = wal;  // published to the consumers by the arrive below
                pmb = (uint32_t)(TYv * NL.mp * 4);
                wnb = (uint32_t)((wae - wal) * (int)sizeof(T));
                extra = pmb + wnb;
            }
            mbar_expect_tx(&full[st], total + extra);
            T* tile = tile_of(st);
            const T* plane = xc + (long long)z * G.plane;
            for (int q = 0; q < nruns; ++q)
                bulk_g2s(tile + run_t[q] * nxp, plane + (long long)run_y[q] * nxp, run_n[q] * rowb, &full[st]);
            const long long own0 = (long long)z * G.plane + (long long)y0 * nxp;
            if (XOLD) bulk_g2s(xold_of(st), xoc + own0, ownb, &full[st]);
            bulk_g2s(veff_of(st), V + own0, vb, &full[st]);
            if constexpr (NLF) {
                bulk_g2s(pm_of(st), NL.ptmap + ((long long)z * ny + y0) * NL.mp, pmb, &full[st]);
                if (wnb) bulk_g2s(wnl_of(st), NL.W + col * NL.ldw + wal, wnb, &full[st]);
            }
            // rows of the plane that enters the consumers' z-window after iteration i
            if (i + 1 < nplanes) {
                const int wst = i % DW, wk = i / DW;
                if (wk > 0 && !mbar_wait(&wempty[wst], (uint32_t)((wk - 1) & 1))) {
                    atomicExch(err, 1);
                    return;
                }
                int zw = z + R + 1;
                zw -= (zw >= nz) ? nz : 0;
                mbar_expect_tx(&wfull[wst], ownb);
                bulk_g2s(wstage_of(wst), xc + (long long)zw * G.plane + (long long)y0 * nxp, ownb, &wfull[wst]);
            }
        }
        return;
    }

    // ------------------------------ consumer warps ------------------------------
    const int lane = tid & 31;
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
    // x-neighbour vectors: start columns wrapped into [0, nx) (nx is a multiple of RX, so a
    // vector never straddles the boundary); bit 2k / 2k+1 of xwrap: vector k wrapped left/right.
    int xcol[NXV];
    unsigned xwrap = 0;
#pragma unroll
    for (int k = 0; k < NXV; ++k) {
        int c = xb - XOFF + k * RX;
        if (c < 0) {
            c += nx;
            xwrap |= 1u << (2 * k);
        } else if (c >= nx) {
            c -= nx;
            xwrap |= 2u << (2 * k);
        }
        xcol[k] = c;
    }
    // y neighbours row R + yl +- p (staged rows); bit (r*2R + 2(p-1)) / +1: the row above / below
    // was copied across the y boundary (top rows wrap left, bottom rows wrap right).
    unsigned long long ywrap = 0;
    if (PHASED) {
#pragma unroll
        for (int r = 0; r < RY; ++r)
#pragma unroll
            for (int p = 1; p <= R; ++p) {
                if (y0 + yl[r] + p >= ny) ywrap |= 1ull << (r * 2 * R + 2 * (p - 1));
                if (y0 + yl[r] - p < 0) ywrap |= 2ull << (r * 2 * R + 2 * (p - 1));
            }
    }

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
        const T* base = xc + (long long)zz * G.plane + (long long)y0 * nxp + xb;
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            VT t;
            if (own[r]) {
                t = *reinterpret_cast<const VT*>(base + (long long)yl[r] * nxp);
            } else {
                T* tp = reinterpret_cast<T*>(&t);
#pragma unroll
                for (int u = 0; u < RX; ++u) tp[u] = zero;
            }
            if (wrapped) {
                T* tp = reinterpret_cast<T*>(&t);
#pragma unroll
                for (int u = 0; u < RX; ++u) tp[u] = pmul(tp[u], mul);
            }
            v[r] = t;
        }
    };

    // y neighbours of the thread's rows: staged rows R + yl[0] + q, q in [-R, RY-1+R].
    // PHASED: bit (q+R) of ywrap_l / ywrap_r: that row was copied across the lower / upper y boundary.
    unsigned ywrap_l = 0, ywrap_r = 0;
    if (PHASED) {
#pragma unroll
        for (int q = -R; q < RY + R; ++q) {
            const int gy = y0 + yl[0] + q;
            if (gy < 0) ywrap_l |= 1u << (q + R);
            else if (gy >= ny) ywrap_r |= 1u << (q + R);
        }
    }

    // z-window: 2R+2 slots so that two planes are marched per loop trip (slot j+k holds
    // plane z-R+k for the plane z handled at sub-step j); sliding by two halves the moves.
    VT w[W + 1][RY];
#pragma unroll
    for (int k = 0; k < W; ++k) load_own_plane(z0 - R + k, w[k]);

    // Entering plane of the window (plane z+R+1 after sub-step i), from the window ring.
    // Per-thread byte offsets in the staged rows (pitch nxp): rowb per row, yoffb to the
    // thread's first point in row yl[0] of a block of own rows, soffb the same for the Veff
    // rows (scalar type S), xcolb the thread's x-neighbour vectors; othr: the thread's first
    // output point of the chunk's first plane.
    const uint32_t rowb = (uint32_t)(nxp * (int)sizeof(T));
    const uint32_t rowbS = (uint32_t)(nxp * (int)sizeof(S));
    const uint32_t yoffb = (uint32_t)((yl[0] * nxp + xb) * (int)sizeof(T));
    const uint32_t soffb = (uint32_t)((yl[0] * nxp + xb) * (int)sizeof(S));
    uint32_t xcolb[NXV];
#pragma unroll
    for (int k = 0; k < NXV; ++k) xcolb[k] = (uint32_t)(xcol[k] * (int)sizeof(T));
    T* const othr = oc + (long long)z0 * G.plane + (long long)(y0 + yl[0]) * nxp + xb;

    auto window_entry = [&](int i, int z, VT* dst) -> bool {
        const int wst = i % DW;
        if (!mbar_wait(&wfull[wst], (uint32_t)((i / DW) & 1))) return false;
        const uint32_t wsrc = smem_u32(wstage_of(wst)) + yoffb;
        const bool wrapped = (z + R + 1) >= nz;
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            VT t;
            if (own[r]) {
                t = lds<VT>(wsrc + r * rowb);
                if (wrapped) {
                    T* tp = reinterpret_cast<T*>(&t);
#pragma unroll
                    for (int u = 0; u < RX; ++u) tp[u] = pmul(tp[u], C.phr[2]);
                }
            } else {
                T* tp = reinterpret_cast<T*>(&t);
#pragma unroll
                for (int u = 0; u < RX; ++u) tp[u] = zero;
            }
            dst[r] = t;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&wempty[wst]);
        return true;
    };

    // FP32 with RX = 2: the same sums in packed FP32x2 arithmetic (fma.rn.f32x2 / add / mul).
    // Every output element sees exactly the scalar path's operations in the same order, so the
    // results are bitwise identical; the instruction count of the z, y, V and x_old terms and of
    // the even x offsets halves.
    auto packed_plane = [&](auto Jc, int z, int st, const T* tile, const T* xo_s, const S* v_s) {
        if constexpr (kPacked) {
            constexpr int J = decltype(Jc)::value;
            float2 acc[RY];
            // fused nonlocal term: this plane's point map at the thread's first row and the staged
            // W range, shifted so that a compact point number indexes it directly
            uint32_t nl_pm = 0, nl_w = 0;
            if constexpr (NLF) {
                nl_pm = smem_u32(pm_of(st)) + (uint32_t)((yl[0] * NL.mp + xb) * 4);
                nl_w = smem_u32(wnl_of(st)) - (uint32_t)walign[st] * 4u;
            }
            const float2 dg = make_float2(C.diag, C.diag);
            const float2 dgl = make_float2(C.diag_lo, C.diag_lo);
            // the neighbour sums first and the (large) centre term last: accumulated from the centre
            // on, the sum would sit at ~40 Ha x, where the rounding loses the centre's lo part and
            // shifts the whole spectrum
#pragma unroll
            for (int r = 0; r < RY; ++r) {
                acc[r] = __fmul2_rn(make_float2(C.cz[1], C.cz[1]), __fadd2_rn(w[J + R + 1][r], w[J + R - 1][r]));
#pragma unroll
                for (int p = 2; p <= R; ++p)
                    acc[r] = __ffma2_rn(make_float2(C.cz[p], C.cz[p]), __fadd2_rn(w[J + R + p][r], w[J + R - p][r]),
                                        acc[r]);
            }
            {
                uint32_t ya = smem_u32(tile) + yoffb;  // row R + yl[0] + q for q = -R
#pragma unroll
                for (int q = -R; q < RY + R; ++q) {
                    float2 v = lds<float2>(ya);
                    ya += rowb;
                    if (PHASED) {
                        if (ywrap_l & (1u << (q + R))) {
                            v.x *= C.phl[1];
                            v.y *= C.phl[1];
                        } else if (ywrap_r & (1u << (q + R))) {
                            v.x *= C.phr[1];
                            v.y *= C.phr[1];
                        }
                    }
#pragma unroll
                    for (int r = 0; r < RY; ++r) {
                        const int d = (q > r) ? q - r : r - q;
                        if (d >= 1 && d <= R) acc[r] = __ffma2_rn(make_float2(C.cy[d], C.cy[d]), v, acc[r]);
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < RY; ++r) {
                if (!own[r]) continue;
                const uint32_t ra = smem_u32(tile) + (uint32_t)(R + yl[r]) * rowb;
                float2 P[NXV];
#pragma unroll
                for (int k = 0; k < NXV; ++k) {
                    float2 t = lds<float2>(ra + xcolb[k]);
                    if (PHASED) {
                        if (xwrap & (1u << (2 * k))) {
                            t.x *= C.phl[0];
                            t.y *= C.phl[0];
                        } else if (xwrap & (2u << (2 * k))) {
                            t.x *= C.phr[0];
                            t.y *= C.phr[0];
                        }
                    }
                    P[k] = t;
                }
                constexpr int H = XOFF / 2;
#pragma unroll
                for (int p = 1; p <= R; ++p) {
                    if (p % 2 == 0) {
                        acc[r] = __ffma2_rn(make_float2(C.cx[p], C.cx[p]), __fadd2_rn(P[H + p / 2], P[H - p / 2]), acc[r]);
                    } else {
                        const float2 sl = __fadd2_rn(P[(XOFF - 1 + p) / 2], P[(XOFF - 1 - p) / 2]);
                        const float2 sr = __fadd2_rn(P[(XOFF + 1 + p) / 2], P[(XOFF + 1 - p) / 2]);
                        acc[r].x = fmaf(C.cx[p], sl.y, acc[r].x);
                        acc[r].y = fmaf(C.cx[p], sr.x, acc[r].y);
                    }
                }
                acc[r] = __ffma2_rn(dgl, w[J + R][r], __ffma2_rn(dg, w[J + R][r], acc[r]));
                const float2 vv = lds<float2>(smem_u32(v_s) + soffb + r * rowbS);
                acc[r] = __ffma2_rn(__fmul2_rn(make_float2(C.a, C.a), vv), w[J + R][r], acc[r]);
                if (XOLD) acc[r] = __ffma2_rn(make_float2(C.d, C.d), lds<float2>(smem_u32(xo_s) + yoffb + r * rowb), acc[r]);
                if constexpr (NLF) {
                    const int2 m = lds<int2>(nl_pm + (uint32_t)r * (uint32_t)(NL.mp * 4));
                    if (m.x >= 0) acc[r].x = fmaf(C.a, lds<float>(nl_w + (uint32_t)m.x * 4u), acc[r].x);
                    if (m.y >= 0) acc[r].y = fmaf(C.a, lds<float>(nl_w + (uint32_t)m.y * 4u), acc[r].y);
                    if (NL.xs_out) {
                        float* xs = NL.xs_out + col * NL.ldw;
                        if (m.x >= 0) xs[m.x] = acc[r].x;
                        if (m.y >= 0) xs[m.y] = acc[r].y;
                    }
                }
                float* op = othr + (long long)(z - z0) * G.plane + r * nxp;
                *reinterpret_cast<float2*>(op) = acc[r];
            }
        }
    };

    // One plane with the window starting at slot J.
    auto plane_step = [&](auto Jc, int i) -> bool {
        constexpr int J = decltype(Jc)::value;
        const int z = z0 + i;
        const int st = i % NS;
        if (!mbar_wait(&full[st], (uint32_t)((i / NS) & 1))) return false;
        const T* tile = tile_of(st);
        const T* xo_s = XOLD ? xold_of(st) : nullptr;
        const S* v_s = veff_of(st);
        if constexpr (kPacked) {
            packed_plane(Jc, z, st, tile, xo_s, v_s);
        } else {
        T acc[RY][RX];
        // centre, z neighbours
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            const T* wc = reinterpret_cast<const T*>(&w[J + R][r]);
            {  // neighbour sums first, the centre term last (see the packed path)
                const T* a_ = reinterpret_cast<const T*>(&w[J + R + 1][r]);
                const T* b_ = reinterpret_cast<const T*>(&w[J + R - 1][r]);
#pragma unroll
                for (int u = 0; u < RX; ++u) acc[r][u] = vscale(C.cz[1], vadd(a_[u], b_[u]));
            }
#pragma unroll
            for (int p = 2; p <= R; ++p) {
                const T* a_ = reinterpret_cast<const T*>(&w[J + R + p][r]);
                const T* b_ = reinterpret_cast<const T*>(&w[J + R - p][r]);
#pragma unroll
                for (int u = 0; u < RX; ++u) acc[r][u] = fmac(acc[r][u], C.cz[p], vadd(a_[u], b_[u]));
            }
        }
        // y neighbours: each staged row is read once and feeds every row within R of it
        {
            uint32_t ya = smem_u32(tile) + yoffb;  // row R + yl[0] + q for q = -R
#pragma unroll
            for (int q = -R; q < RY + R; ++q) {
                VT v = lds<VT>(ya);
                ya += rowb;
                T* ve = reinterpret_cast<T*>(&v);
                if (PHASED) {
                    if (ywrap_l & (1u << (q + R))) {
#pragma unroll
                        for (int u = 0; u < RX; ++u) ve[u] = pmul(ve[u], C.phl[1]);
                    } else if (ywrap_r & (1u << (q + R))) {
#pragma unroll
                        for (int u = 0; u < RX; ++u) ve[u] = pmul(ve[u], C.phr[1]);
                    }
                }
#pragma unroll
                for (int r = 0; r < RY; ++r) {
                    const int d = (q > r) ? q - r : r - q;
                    if (d >= 1 && d <= R) {
#pragma unroll
                        for (int u = 0; u < RX; ++u) acc[r][u] = fmac(acc[r][u], C.cy[d], ve[u]);
                    }
                }
            }
        }
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            if (!own[r]) continue;
            const uint32_t ra = smem_u32(tile) + (uint32_t)(R + yl[r]) * rowb;
            // x neighbours
            {
                T xv[NXV * RX];
#pragma unroll
                for (int k = 0; k < NXV; ++k) {
                    VT t = lds<VT>(ra + xcolb[k]);
                    if (PHASED) {
                        T* tp = reinterpret_cast<T*>(&t);
                        if (xwrap & (1u << (2 * k))) {
#pragma unroll
                            for (int u = 0; u < RX; ++u) tp[u] = pmul(tp[u], C.phl[0]);
                        } else if (xwrap & (2u << (2 * k))) {
#pragma unroll
                            for (int u = 0; u < RX; ++u) tp[u] = pmul(tp[u], C.phr[0]);
                        }
                    }
                    *reinterpret_cast<VT*>(&xv[k * RX]) = t;
                }
#pragma unroll
                for (int u = 0; u < RX; ++u)
#pragma unroll
                    for (int p = 1; p <= R; ++p)
                        acc[r][u] = fmac(acc[r][u], C.cx[p], vadd(xv[XOFF + u + p], xv[XOFF + u - p]));
            }
            const T* wc = reinterpret_cast<const T*>(&w[J + R][r]);
            {
                S vv[RX];
                const uint32_t va = smem_u32(v_s) + soffb + r * rowbS;
                if constexpr (RX == 2) {
                    using SV = typename VecOf<S, 2>::type;
                    *reinterpret_cast<SV*>(vv) = lds<SV>(va);
                } else {
                    vv[0] = lds<S>(va);
                }
                VT xo_v;
                if (XOLD) xo_v = lds<VT>(smem_u32(xo_s) + yoffb + r * rowb);
                const T* xo_e = reinterpret_cast<const T*>(&xo_v);
#pragma unroll
                for (int u = 0; u < RX; ++u) {
                    acc[r][u] = fmac(acc[r][u], C.diag, wc[u]);
                    if (sizeof(S) == sizeof(float)) acc[r][u] = fmac(acc[r][u], C.diag_lo, wc[u]);
                    acc[r][u] = fmac(acc[r][u], C.a * vv[u], wc[u]);
                    if (XOLD) acc[r][u] = fmac(acc[r][u], C.d, xo_e[u]);
                }
            }
            if constexpr (NLF) {
                const int* pmr = pm_of(st) + yl[r] * NL.mp + xb;
                const T* wn = wnl_of(st) - walign[st];
#pragma unroll
                for (int u = 0; u < RX; ++u) {
                    const int m = pmr[u];
                    if (m >= 0) {
                        acc[r][u] = fmac(acc[r][u], C.a, wn[m]);
                        if (NL.xs_out) NL.xs_out[col * NL.ldw + m] = acc[r][u];
                    }
                }
            }
            T* op = othr + (long long)(z - z0) * G.plane + r * nxp;
            VT o;
            T* opv = reinterpret_cast<T*>(&o);
#pragma unroll
            for (int u = 0; u < RX; ++u) opv[u] = acc[r][u];
            *reinterpret_cast<VT*>(op) = o;
        }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[st]);
        return true;
    };

    bool ok = true;
    for (int i = 0; i < nplanes && ok; i += 2) {
        // sub-step 0: plane i, window slots 0..2R
        ok = plane_step(std::integral_constant<int, 0>{}, i);
        if (!ok || i + 1 >= nplanes) break;
        ok = window_entry(i, z0 + i, w[W]);  // plane i+R+1 -> slot 2R+1
        if (!ok) break;
        // sub-step 1: plane i+1, window slots 1..2R+1
        ok = plane_step(std::integral_constant<int, 1>{}, i + 1);
        if (!ok || i + 2 >= nplanes) break;
        // slide by two and bring in plane i+R+2
#pragma unroll
        for (int k = 0; k < W - 1; ++k)
#pragma unroll
            for (int r = 0; r < RY; ++r) w[k][r] = w[k + 2][r];
        ok = window_entry(i + 1, z0 + i + 1, w[W - 1]);
    }
    if (!ok && lane == 0) atomicExch(err, 1);
}

}  // namespace lynxb
