// Launch-shape selection and template dispatch for the fused Chebyshev-step kernel.
// Compiled once per value type (LYNX_STENCIL_TYPES selects real or complex) so the
// instantiations build in parallel.
#include <algorithm>
#include <cstdio>
#include <type_traits>

#include "kernels.h"
#include "lynx_common.cuh"
#include "stencil.cuh"

namespace lynxb {

namespace {

template <typename T> constexpr int rows_per_thread() { return ScalarOf<T>::cplx ? 1 : 2; }

template <typename T, int R, int HK, bool XOLD>
void launch_one(dim3 grid, int nthr, size_t smem, cudaStream_t st, const T* x, const T* xold, T* out,
                const typename ScalarOf<T>::type* V, const StencilArgs<T>& A) {
    constexpr int RY = rows_per_thread<T>();
    auto kern = cheb_step_kernel<T, R, RY, HK, XOLD>;
    smem_cap(kern, smem);
    kern<<<grid, nthr, smem, st>>>(x, xold, out, V, A);
}

template <typename T, int R>
int dispatch_r(int HK, bool xold, dim3 grid, int nthr, size_t smem, cudaStream_t st, const T* x,
               const T* xo, T* out, const typename ScalarOf<T>::type* V, const StencilArgs<T>& A) {
    if (HK <= 4) {
        if (xold) launch_one<T, R, 4, true>(grid, nthr, smem, st, x, xo, out, V, A);
        else launch_one<T, R, 4, false>(grid, nthr, smem, st, x, xo, out, V, A);
    } else {
        if (xold) launch_one<T, R, 8, true>(grid, nthr, smem, st, x, xo, out, V, A);
        else launch_one<T, R, 8, false>(grid, nthr, smem, st, x, xo, out, V, A);
    }
    return 0;
}

}  // namespace

template <typename T, typename S>
int launch_cheb_step(const StencilGeom& g, const T* x, long long ldx, const T* xold, long long ldo, T* out,
                     long long ldout, const S* V, int ncol, double a, double b, double d, const T* phl,
                     const T* phr, cudaStream_t st) {
    static_assert(std::is_same<S, typename ScalarOf<T>::type>::value, "scalar type mismatch");
    const int R = g.R;
    if (R < 1 || R > 8) {
        set_error("FD half-width %d outside the supported range 1..8", R);
        return LYNX_ERR_UNSUPPORTED;
    }
    if (g.nx < R || g.ny < R || g.nz < R) {
        set_error("grid %dx%dx%d smaller than the FD half-width %d", g.nx, g.ny, g.nz, R);
        return LYNX_ERR_UNSUPPORTED;
    }
    if (g.nx > kStencilMaxThreads) {
        set_error("nx = %d above the supported maximum %d", g.nx, kStencilMaxThreads);
        return LYNX_ERR_UNSUPPORTED;
    }
    if (ncol <= 0) return LYNX_OK;
    constexpr int RY = rows_per_thread<T>();
    // Thread rows: aim at ~288 threads per CTA, whole x-rows per thread row.
    int TYT = std::max(1, (288 + g.nx / 2) / g.nx);
    TYT = std::min(TYT, kStencilMaxThreads / g.nx);
    TYT = std::min(TYT, (g.ny + RY - 1) / RY);
    const int nthr = ((g.nx * TYT + 31) / 32) * 32;
    const int HK = (2 * R * g.nx + nthr - 1) / nthr;
    if (HK > 8) {
        set_error("halo of %d elements per plane too large for %d threads", 2 * R * g.nx, nthr);
        return LYNX_ERR_UNSUPPORTED;
    }
    StencilArgs<T> A;
    A.nx = g.nx;
    A.ny = g.ny;
    A.nz = g.nz;
    A.ld_x = ldx;
    A.ld_old = ldo;
    A.ld_out = ldout;
    A.TYT = TYT;
    A.TY = TYT * RY;
    const int nbands = (g.ny + A.TY - 1) / A.TY;
    // Enough CTAs to fill the machine: split z when bands x columns are few.
    const long long base = (long long)nbands * ncol;
    int nzch = (int)std::min<long long>((1200 + base - 1) / base, std::max(1, g.nz / (4 * R)));
    nzch = std::max(1, nzch);
    A.zchunk = (g.nz + nzch - 1) / nzch;
    nzch = (g.nz + A.zchunk - 1) / A.zchunk;
    for (int p = 0; p <= 8; ++p) {
        A.cx[p] = A.cy[p] = A.cz[p] = S(0);
    }
    for (int p = 1; p <= R; ++p) {
        A.cx[p] = (S)(-0.5 * a * g.D2x[p]);
        A.cy[p] = (S)(-0.5 * a * g.D2y[p]);
        A.cz[p] = (S)(-0.5 * a * g.D2z[p]);
    }
    centre_coef<S>(g, a, b, A.cx, A.cy, A.cz, &A.diag, &A.diag_lo);
    A.a = (S)a;
    A.d = (S)d;
    for (int k = 0; k < 3; ++k) {
        A.phl[k] = phl[k];
        A.phr[k] = phr[k];
    }
    const size_t smem = (size_t)(A.TY + 2 * R) * (g.nx + 2 * R) * sizeof(T);
    if (smem > 200 * 1024) {
        set_error("staging plane of %zu bytes exceeds shared memory", smem);
        return LYNX_ERR_UNSUPPORTED;
    }
    if (ncol > 65535 || nzch > 65535) {
        set_error("too many columns (%d) for one launch", ncol);
        return LYNX_ERR_UNSUPPORTED;
    }
    dim3 grid(nbands, ncol, nzch);
    const bool xo = (xold != nullptr) && d != 0.0;
    switch (R) {
        case 1: dispatch_r<T, 1>(HK, xo, grid, nthr, smem, st, x, xold, out, V, A); break;
        case 2: dispatch_r<T, 2>(HK, xo, grid, nthr, smem, st, x, xold, out, V, A); break;
        case 3: dispatch_r<T, 3>(HK, xo, grid, nthr, smem, st, x, xold, out, V, A); break;
        case 4: dispatch_r<T, 4>(HK, xo, grid, nthr, smem, st, x, xold, out, V, A); break;
        case 5: dispatch_r<T, 5>(HK, xo, grid, nthr, smem, st, x, xold, out, V, A); break;
        case 6: dispatch_r<T, 6>(HK, xo, grid, nthr, smem, st, x, xold, out, V, A); break;
        case 7: dispatch_r<T, 7>(HK, xo, grid, nthr, smem, st, x, xold, out, V, A); break;
        case 8: dispatch_r<T, 8>(HK, xo, grid, nthr, smem, st, x, xold, out, V, A); break;
    }
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("stencil launch failed: %s", cudaGetErrorString(e));
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

#if LYNX_STENCIL_TYPES == 0
template int launch_cheb_step<double, double>(const StencilGeom&, const double*, long long, const double*,
                                              long long, double*, long long, const double*, int, double,
                                              double, double, const double*, const double*, cudaStream_t);
template int launch_cheb_step<float, float>(const StencilGeom&, const float*, long long, const float*,
                                            long long, float*, long long, const float*, int, double, double,
                                            double, const float*, const float*, cudaStream_t);
#else
template int launch_cheb_step<double2, double>(const StencilGeom&, const double2*, long long, const double2*,
                                               long long, double2*, long long, const double*, int, double,
                                               double, double, const double2*, const double2*, cudaStream_t);
template int launch_cheb_step<float2, float>(const StencilGeom&, const float2*, long long, const float2*,
                                             long long, float2*, long long, const float*, int, double, double,
                                             double, const float2*, const float2*, cudaStream_t);
#endif

}  // namespace lynxb
