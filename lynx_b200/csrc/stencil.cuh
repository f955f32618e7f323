// Fused Chebyshev-filter step for sm_100a:
//   out = a * (-0.5 * Lap x + Veff .* x) + b * x + d * xold
// on a 3-D grid with the ghost values produced inside the kernel (periodic wrap,
// Bloch phase e^{+-i k_d L_d}, or zero for Dirichlet) — no padded copy of x is
// ever written.  One launch does one degree step of the filter
// (src/solvers/EigenSolver.cpp:586-607 recurrence, src/operators/Hamiltonian.cpp:127-174
// stencil, src/parallel/HaloExchange.cpp:34-95 ghost rules).
//
// Work decomposition.  A CTA owns one orbital column, a band of TY full x-rows
// (all nx points of each row) and a chunk of z-planes, and marches through the
// chunk one z-plane at a time:
//   - the z-direction neighbours of every owned point live in a register window
//     of 2R+1 planes that slides with the march (each plane of x is read from
//     HBM once per CTA);
//   - the current plane's owned rows plus R halo rows above/below the band are
//     staged in shared memory with R ghost columns on each side, so the x- and
//     y-direction neighbours are shared-memory reads;
//   - the x ghosts are written by the threads that own the wrapped points
//     (duplicate stores), so periodic x needs no extra loads;
//   - the next plane's window value, halo rows, xold and Veff are prefetched
//     into registers one plane ahead, so their latency overlaps the current
//     plane's arithmetic.
// HBM traffic per update is x (once), xold (once), out (once): 3 words, the
// algorithmic floor.  Halo rows and Veff are re-read from L2.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace lynxb {

template <typename T> struct ScalarOf;
template <> struct ScalarOf<double> { using type = double; static constexpr bool cplx = false; };
template <> struct ScalarOf<float> { using type = float; static constexpr bool cplx = false; };
template <> struct ScalarOf<double2> { using type = double; static constexpr bool cplx = true; };
template <> struct ScalarOf<float2> { using type = float; static constexpr bool cplx = true; };

__device__ __forceinline__ double vzero(double) { return 0.0; }
__device__ __forceinline__ float vzero(float) { return 0.0f; }
__device__ __forceinline__ double2 vzero(double2) { return make_double2(0.0, 0.0); }
__device__ __forceinline__ float2 vzero(float2) { return make_float2(0.0f, 0.0f); }

// acc + c * v  (c real)
__device__ __forceinline__ double fmac(double acc, double c, double v) { return fma(c, v, acc); }
__device__ __forceinline__ float fmac(float acc, float c, float v) { return fmaf(c, v, acc); }
__device__ __forceinline__ double2 fmac(double2 acc, double c, double2 v) {
    return make_double2(fma(c, v.x, acc.x), fma(c, v.y, acc.y));
}
__device__ __forceinline__ float2 fmac(float2 acc, float c, float2 v) {
    return make_float2(fmaf(c, v.x, acc.x), fmaf(c, v.y, acc.y));
}
__device__ __forceinline__ double vadd(double a, double b) { return a + b; }
__device__ __forceinline__ float vadd(float a, float b) { return a + b; }
__device__ __forceinline__ double2 vadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double vscale(double c, double v) { return c * v; }
__device__ __forceinline__ float vscale(float c, float v) { return c * v; }
__device__ __forceinline__ double2 vscale(double c, double2 v) { return make_double2(c * v.x, c * v.y); }
__device__ __forceinline__ float2 vscale(float c, float2 v) { return make_float2(c * v.x, c * v.y); }
// v * ph: real phase for real data, complex product for complex data.
__device__ __forceinline__ double pmul(double v, double ph) { return v * ph; }
__device__ __forceinline__ float pmul(float v, float ph) { return v * ph; }
__device__ __forceinline__ double2 pmul(double2 v, double2 ph) {
    return make_double2(v.x * ph.x - v.y * ph.y, v.x * ph.y + v.y * ph.x);
}
__device__ __forceinline__ float2 pmul(float2 v, float2 ph) {
    return make_float2(v.x * ph.x - v.y * ph.y, v.x * ph.y + v.y * ph.x);
}

constexpr int kStencilMaxThreads = 512;

template <typename T>
struct StencilArgs {
    using S = typename ScalarOf<T>::type;
    int nx, ny, nz;
    long long ld_x, ld_old, ld_out;  // column strides (elements of T)
    int TYT;     // thread rows per CTA
    int TY;      // band height = TYT * RY
    int zchunk;  // z-planes per CTA
    S cx[9], cy[9], cz[9];  // cx[p] = -0.5 * a * D2_x[p], p = 1..R
    S diag, diag_lo;        // -0.5 * a * (D2_x[0] + D2_y[0] + D2_z[0]) + b as a (hi, lo) pair (centre_coef)
    S a;                    // multiplies Veff .* x
    S d;                    // multiplies xold
    T phl[3], phr[3];       // multipliers of left / right ghosts per direction (1, 0 or Bloch phase)
};

// HK: halo elements per thread per plane (2R*nx <= HK*blockDim).
template <typename T, int R, int RY, int HK, bool XOLD>
__global__ void __launch_bounds__(kStencilMaxThreads)
    cheb_step_kernel(const T* __restrict__ x, const T* __restrict__ xold, T* __restrict__ out,
                     const typename ScalarOf<T>::type* __restrict__ V, const StencilArgs<T> A) {
    using S = typename ScalarOf<T>::type;
    constexpr int W = 2 * R + 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* sm = reinterpret_cast<T*>(smraw);

    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const long long nxny = (long long)nx * ny;
    const int y0 = blockIdx.x * A.TY;
    const int TYv = min(A.TY, ny - y0);
    const int z0 = blockIdx.z * A.zchunk;
    const int z1 = min(nz, z0 + A.zchunk);
    const long long col = blockIdx.y;
    const T* __restrict__ xc = x + col * A.ld_x;
    const T* __restrict__ xoc = XOLD ? (xold + col * A.ld_old) : nullptr;
    T* __restrict__ oc = out + col * A.ld_out;

    const int pitch = nx + 2 * R;
    const int tid = threadIdx.x;
    const int nthr = blockDim.x;
    const int tx = tid % nx;
    const int ty = tid / nx;
    const T zero = vzero(T());

    int yl[RY];
    bool own[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        yl[r] = ty * RY + r;
        own[r] = (ty < A.TYT) && (yl[r] < TYv);
    }

    // Zero the staging plane once: ghost cells that a Dirichlet boundary never writes stay zero.
    const int smsize = (A.TY + 2 * R) * pitch;
    for (int i = tid; i < smsize; i += nthr) sm[i] = zero;

    // Halo rows of the band (R above, R below), assigned round-robin to threads.
    // Packed per element: smem index (low 20 bits), wrap code (bits 20-21:
    // 0 none, 1 left wrap, 2 right wrap, 3 not assigned), ghost code (bits 22-23:
    // 1 also write the right x-ghost, 2 also write the left x-ghost).  A
    // Dirichlet boundary is a wrap whose multiplier is 0.
    const int nh = 2 * R * nx;
    int h_goff[HK];
    int h_info[HK];
#pragma unroll
    for (int k = 0; k < HK; ++k) {
        const int h = tid + k * nthr;
        h_goff[k] = 0;
        h_info[k] = 3 << 20;
        if (h < nh) {
            const int hr = h / nx;
            const int hx = h - hr * nx;
            int gy, srow;
            if (hr < R) {
                gy = y0 - R + hr;
                srow = hr;
            } else {
                gy = y0 + TYv + (hr - R);
                srow = TYv + hr;
            }
            int wrap = 0;
            if (gy < 0) {
                gy += ny;
                wrap = 1;
            } else if (gy >= ny) {
                gy -= ny;
                wrap = 2;
            }
            const int ghost = (hx < R) ? 1 : ((hx >= nx - R) ? 2 : 0);
            h_goff[k] = gy * nx + hx;
            h_info[k] = (srow * pitch + hx + R) | (wrap << 20) | (ghost << 22);
        }
    }
    const T phl_y = A.phl[1], phr_y = A.phr[1];

    auto load_halo = [&](int z, T* hv) {
        const T* plane = xc + (long long)z * nxny;
#pragma unroll
        for (int k = 0; k < HK; ++k) {
            const int wrap = (h_info[k] >> 20) & 3;
            T v = zero;
            if (wrap != 3) {
                v = __ldg(plane + h_goff[k]);
                if (wrap == 1) v = pmul(v, phl_y);
                else if (wrap == 2) v = pmul(v, phr_y);
            }
            hv[k] = v;
        }
    };
    auto load_own = [&](int zz, T* v) {
        T mul = A.phl[2];
        bool wrapped = false;
        if (zz < 0) {
            zz += nz;
            wrapped = true;
        } else if (zz >= nz) {
            zz -= nz;
            mul = A.phr[2];
            wrapped = true;
        }
        const T* plane = xc + (long long)zz * nxny + (long long)y0 * nx + tx;
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            T t = own[r] ? __ldg(plane + yl[r] * nx) : zero;
            v[r] = wrapped ? pmul(t, mul) : t;
        }
    };

    // Register window: w[k][r] = x at plane (z - R + k), owned row r.
    T w[W][RY];
#pragma unroll
    for (int k = 0; k < W; ++k) load_own(z0 - R + k, w[k]);
    T hcur[HK], hnxt[HK];
    load_halo(z0, hcur);
    T xo_cur[RY], xo_nxt[RY];
    S v_cur[RY], v_nxt[RY];
    {
        const long long base = (long long)z0 * nxny + (long long)y0 * nx + tx;
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            const long long o = base + yl[r] * nx;
            xo_cur[r] = (XOLD && own[r]) ? __ldg(xoc + o) : zero;
            v_cur[r] = own[r] ? __ldg(V + o) : S(0);
        }
    }
    __syncthreads();  // staging plane zeroed

    const T phl_x = A.phl[0], phr_x = A.phr[0];
    for (int z = z0; z < z1; ++z) {
        // Prefetch everything the next plane needs.
        T nxt[RY];
        if (z + 1 < z1) {
            load_own(z + R + 1, nxt);
            load_halo(z + 1, hnxt);
            const long long base = (long long)(z + 1) * nxny + (long long)y0 * nx + tx;
#pragma unroll
            for (int r = 0; r < RY; ++r) {
                const long long o = base + yl[r] * nx;
                xo_nxt[r] = (XOLD && own[r]) ? __ldg(xoc + o) : zero;
                v_nxt[r] = own[r] ? __ldg(V + o) : S(0);
            }
        }
        __syncthreads();  // S1: previous plane's reads of sm are done
        // Owned rows of plane z, plus their x-ghost images.
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            if (own[r]) {
                const int si = (R + yl[r]) * pitch + tx + R;
                const T v = w[R][r];
                sm[si] = v;
                if (tx < R) sm[si + nx] = pmul(v, phr_x);
                if (tx >= nx - R) sm[si - nx] = pmul(v, phl_x);
            }
        }
        // Halo rows of plane z, plus their x-ghost images.
#pragma unroll
        for (int k = 0; k < HK; ++k) {
            if (tid + k * nthr < nh) {
                const int info = h_info[k];
                const int si = info & 0xFFFFF;
                const int ghost = (info >> 22) & 3;
                const T v = hcur[k];
                sm[si] = v;
                if (ghost == 1) sm[si + nx] = pmul(v, phr_x);
                else if (ghost == 2) sm[si - nx] = pmul(v, phl_x);
            }
        }
        __syncthreads();  // S2: plane z staged

        const long long obase = (long long)z * nxny + (long long)y0 * nx + tx;
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            if (!own[r]) continue;
            const T* c = sm + (R + yl[r]) * pitch + tx + R;
            // neighbour sums first, the (large) centre term last, so that the accumulator stays
            // small where the centre's lo part is added (FP32: no spectrum-wide shift)
            T acc = vscale(A.cx[1], vadd(c[1], c[-1]));
#pragma unroll
            for (int p = 2; p <= R; ++p) acc = fmac(acc, A.cx[p], vadd(c[p], c[-p]));
#pragma unroll
            for (int p = 1; p <= R; ++p) acc = fmac(acc, A.cy[p], vadd(c[p * pitch], c[-p * pitch]));
#pragma unroll
            for (int p = 1; p <= R; ++p) acc = fmac(acc, A.cz[p], vadd(w[R + p][r], w[R - p][r]));
            acc = fmac(acc, A.diag, w[R][r]);
            if (sizeof(S) == sizeof(float)) acc = fmac(acc, A.diag_lo, w[R][r]);
            acc = fmac(acc, A.a * v_cur[r], w[R][r]);
            if (XOLD) acc = fmac(acc, A.d, xo_cur[r]);
            oc[obase + yl[r] * nx] = acc;
        }

        // Slide the window.
#pragma unroll
        for (int k = 0; k < W - 1; ++k)
#pragma unroll
            for (int r = 0; r < RY; ++r) w[k][r] = w[k + 1][r];
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            w[W - 1][r] = nxt[r];
            xo_cur[r] = xo_nxt[r];
            v_cur[r] = v_nxt[r];
        }
#pragma unroll
        for (int k = 0; k < HK; ++k) hcur[k] = hnxt[k];
    }
}

}  // namespace lynxb
