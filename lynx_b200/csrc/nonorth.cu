// Mixed-derivative terms of the Laplacian on non-orthogonal cells
// (src/operators/Hamiltonian.cpp:177-267, lap_plus_diag_nonorth_impl):
//   Lap += sum_{p,q} c_ab[p] d1_b[q] (x(+pa+qb) - x(+pa-qb) - x(-pa+qb) + x(-pa-qb))
// for (a,b) = (x,y), (x,z), (y,z), with c_ab = D2_coeff_{xy,xz,yz} and d1_b = D1_coeff_{y,z}.
// Evaluated in separable form: first the first derivatives along y and z,
//   gy = sum_q d1_y[q] (x(+qy) - x(-qy)),   gz = sum_q d1_z[q] (x(+qz) - x(-qz)),
// then  mixed = sum_p c_xy[p] (gy(+px) - gy(-px)) + c_xz[p] (gz(+px) - gz(-px))
//             + c_yz[p] (gz(+py) - gz(-py)),
// and out += a * (-1/2) * mixed.  (The same sums in another order: O(R) work per point
// instead of O(R^2).)  Wrapped neighbours carry the ghost multipliers of the periodic / Bloch /
// Dirichlet boundary, as in the stencil kernels; gy and gz are Bloch functions with the same
// multipliers.  Rows have nxp elements (x >= nx is padding and is not written).
#include "kernels.h"
#include "lynx_common.cuh"
#include "stencil.cuh"

namespace lynxb {
namespace {

template <typename T>
struct NOArgs {
    using S = typename ScalarOf<T>::type;
    int nx, ny, nz, nxp, R;
    S d1y[9], d1z[9], cxy[9], cxz[9], cyz[9];
    T phl[3], phr[3];
};

template <typename T>
__device__ __forceinline__ T wrapped(const T* base, long long idx, bool l, bool r, const T& phl, const T& phr) {
    const T v = base[idx];
    if (l) return pmul(v, phl);
    if (r) return pmul(v, phr);
    return v;
}

template <typename T>
__global__ void __launch_bounds__(256)
    nonorth_grad_kernel(const T* __restrict__ x, long long ldx, T* __restrict__ gy, T* __restrict__ gz, long long ldg,
                        const NOArgs<T> A) {
    const long long np = (long long)A.nx * A.ny * A.nz;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int col = blockIdx.y;
    const int i = (int)(t % A.nx);
    const int j = (int)((t / A.nx) % A.ny);
    const int k = (int)(t / ((long long)A.nx * A.ny));
    const T* xb = x + (long long)col * ldx;
    auto at = [&](int ii, int jj, int kk) { return (long long)ii + (long long)A.nxp * (jj + (long long)A.ny * kk); };
    T sy = vzero(T()), sz = vzero(T());
    for (int q = 1; q <= A.R; ++q) {
        int jp = j + q, jm = j - q;
        const bool ry = jp >= A.ny, ly = jm < 0;
        jp -= ry ? A.ny : 0;
        jm += ly ? A.ny : 0;
        const T yp = wrapped(xb, at(i, jp, k), false, ry, A.phl[1], A.phr[1]);
        const T ym = wrapped(xb, at(i, jm, k), ly, false, A.phl[1], A.phr[1]);
        sy = fmac(sy, A.d1y[q], vadd(yp, vscale((typename ScalarOf<T>::type)(-1), ym)));
        int kp = k + q, km = k - q;
        const bool rz = kp >= A.nz, lz = km < 0;
        kp -= rz ? A.nz : 0;
        km += lz ? A.nz : 0;
        const T zp = wrapped(xb, at(i, j, kp), false, rz, A.phl[2], A.phr[2]);
        const T zm = wrapped(xb, at(i, j, km), lz, false, A.phl[2], A.phr[2]);
        sz = fmac(sz, A.d1z[q], vadd(zp, vscale((typename ScalarOf<T>::type)(-1), zm)));
    }
    const long long o = (long long)col * ldg + at(i, j, k);
    gy[o] = sy;
    gz[o] = sz;
}

template <typename T>
__global__ void __launch_bounds__(256)
    nonorth_mixed_kernel(const T* __restrict__ gy, const T* __restrict__ gz, long long ldg, T* __restrict__ out,
                         long long ldout, typename ScalarOf<T>::type scale, const NOArgs<T> A) {
    const long long np = (long long)A.nx * A.ny * A.nz;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int col = blockIdx.y;
    const int i = (int)(t % A.nx);
    const int j = (int)((t / A.nx) % A.ny);
    const int k = (int)(t / ((long long)A.nx * A.ny));
    const T* gyb = gy + (long long)col * ldg;
    const T* gzb = gz + (long long)col * ldg;
    auto at = [&](int ii, int jj, int kk) { return (long long)ii + (long long)A.nxp * (jj + (long long)A.ny * kk); };
    using S = typename ScalarOf<T>::type;
    T m = vzero(T());
    for (int p = 1; p <= A.R; ++p) {
        int ip = i + p, im = i - p;
        const bool rx = ip >= A.nx, lx = im < 0;
        ip -= rx ? A.nx : 0;
        im += lx ? A.nx : 0;
        const T dyx = vadd(wrapped(gyb, at(ip, j, k), false, rx, A.phl[0], A.phr[0]),
                           vscale(S(-1), wrapped(gyb, at(im, j, k), lx, false, A.phl[0], A.phr[0])));
        const T dzx = vadd(wrapped(gzb, at(ip, j, k), false, rx, A.phl[0], A.phr[0]),
                           vscale(S(-1), wrapped(gzb, at(im, j, k), lx, false, A.phl[0], A.phr[0])));
        int jp = j + p, jm = j - p;
        const bool ry = jp >= A.ny, ly = jm < 0;
        jp -= ry ? A.ny : 0;
        jm += ly ? A.ny : 0;
        const T dzy = vadd(wrapped(gzb, at(i, jp, k), false, ry, A.phl[1], A.phr[1]),
                           vscale(S(-1), wrapped(gzb, at(i, jm, k), ly, false, A.phl[1], A.phr[1])));
        m = fmac(m, A.cxy[p], dyx);
        m = fmac(m, A.cxz[p], dzx);
        m = fmac(m, A.cyz[p], dzy);
    }
    T* o = out + (long long)col * ldout + at(i, j, k);
    *o = fmac(*o, scale, m);
}

}  // namespace

template <typename T>
int launch_nonorth_terms(const NonOrthGeom& g, int nxp, const T* x, long long ldx, T* gy, T* gz, long long ldg, T* out,
                         long long ldout, int ncol, double a, const T* phl, const T* phr, cudaStream_t st) {
    using S = typename ScalarOf<T>::type;
    if (g.R < 1 || g.R > 8) {
        set_error("FD half-width %d outside the supported range 1..8", g.R);
        return LYNX_ERR_UNSUPPORTED;
    }
    if (ncol <= 0) return LYNX_OK;
    if (ncol > 65535) {
        set_error("too many columns (%d) for one launch", ncol);
        return LYNX_ERR_UNSUPPORTED;
    }
    NOArgs<T> A;
    A.nx = g.nx;
    A.ny = g.ny;
    A.nz = g.nz;
    A.nxp = nxp;
    A.R = g.R;
    for (int p = 0; p <= 8; ++p) {
        const bool in = p <= g.R;
        A.d1y[p] = in ? (S)g.D1y[p] : S(0);
        A.d1z[p] = in ? (S)g.D1z[p] : S(0);
        A.cxy[p] = in ? (S)g.D2xy[p] : S(0);
        A.cxz[p] = in ? (S)g.D2xz[p] : S(0);
        A.cyz[p] = in ? (S)g.D2yz[p] : S(0);
    }
    for (int d = 0; d < 3; ++d) {
        A.phl[d] = phl[d];
        A.phr[d] = phr[d];
    }
    const long long np = (long long)g.nx * g.ny * g.nz;
    dim3 grid((unsigned)((np + 255) / 256), ncol);
    nonorth_grad_kernel<T><<<grid, 256, 0, st>>>(x, ldx, gy, gz, ldg, A);
    nonorth_mixed_kernel<T><<<grid, 256, 0, st>>>(gy, gz, ldg, out, ldout, (S)(-0.5 * a), A);
    count_launch(2);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("non-orthogonal stencil launch failed: %s", cudaGetErrorString(e));
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

template int launch_nonorth_terms<double>(const NonOrthGeom&, int, const double*, long long, double*, double*, long long,
                                          double*, long long, int, double, const double*, const double*, cudaStream_t);
template int launch_nonorth_terms<float>(const NonOrthGeom&, int, const float*, long long, float*, float*, long long,
                                         float*, long long, int, double, const float*, const float*, cudaStream_t);
template int launch_nonorth_terms<double2>(const NonOrthGeom&, int, const double2*, long long, double2*, double2*,
                                           long long, double2*, long long, int, double, const double2*, const double2*,
                                           cudaStream_t);
template int launch_nonorth_terms<float2>(const NonOrthGeom&, int, const float2*, long long, float2*, float2*,
                                          long long, float2*, long long, int, double, const float2*, const float2*,
                                          cudaStream_t);

}  // namespace lynxb

// ---------------------------------------------------------------------------------------------
// First derivative along one lattice direction (src/operators/Gradient.cpp:17-62):
//   g = sum_p D1[p] (x(+p e_dir) - x(-p e_dir)), ghosts as in the stencil kernels.
// ---------------------------------------------------------------------------------------------
namespace lynxb {
namespace {
template <typename T>
struct GradArgs {
    using S = typename ScalarOf<T>::type;
    int nx, ny, nz, nxp, R, dir;
    S d1[9];
    T phl, phr;
};

template <typename T>
__global__ void __launch_bounds__(256)
    grad_dir_kernel(const T* __restrict__ x, long long ldx, T* __restrict__ g, long long ldg, const GradArgs<T> A) {
    const long long np = (long long)A.nx * A.ny * A.nz;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int col = blockIdx.y;
    const int c[3] = {(int)(t % A.nx), (int)((t / A.nx) % A.ny), (int)(t / ((long long)A.nx * A.ny))};
    const int n[3] = {A.nx, A.ny, A.nz};
    const T* xb = x + (long long)col * ldx;
    auto at = [&](const int* q) { return (long long)q[0] + (long long)A.nxp * (q[1] + (long long)A.ny * q[2]); };
    using S = typename ScalarOf<T>::type;
    T s = vzero(T());
    const int d = A.dir;
    for (int p = 1; p <= A.R; ++p) {
        int q[3] = {c[0], c[1], c[2]};
        int ip = c[d] + p, im = c[d] - p;
        const bool r = ip >= n[d], l = im < 0;
        ip -= r ? n[d] : 0;
        im += l ? n[d] : 0;
        q[d] = ip;
        T vp = xb[at(q)];
        if (r) vp = pmul(vp, A.phr);
        q[d] = im;
        T vm = xb[at(q)];
        if (l) vm = pmul(vm, A.phl);
        s = fmac(s, A.d1[p], vadd(vp, vscale(S(-1), vm)));
    }
    g[(long long)col * ldg + at(c)] = s;
}
}  // namespace

template <typename T>
int launch_grad_dir(int nx, int ny, int nz, int nxp, int R, const double* D1, int dir, const T* x, long long ldx,
                    T* g, long long ldg, int ncol, const T* phl, const T* phr, cudaStream_t st) {
    using S = typename ScalarOf<T>::type;
    if (R < 1 || R > 8 || dir < 0 || dir > 2) {
        set_error("gradient: bad half-width %d or direction %d", R, dir);
        return LYNX_ERR_BAD_ARG;
    }
    if (ncol <= 0) return LYNX_OK;
    if (ncol > 65535) {
        set_error("too many columns (%d) for one launch", ncol);
        return LYNX_ERR_UNSUPPORTED;
    }
    GradArgs<T> A;
    A.nx = nx;
    A.ny = ny;
    A.nz = nz;
    A.nxp = nxp;
    A.R = R;
    A.dir = dir;
    for (int p = 0; p <= 8; ++p) A.d1[p] = (p <= R) ? (S)D1[p] : S(0);
    A.phl = phl[dir];
    A.phr = phr[dir];
    const long long np = (long long)nx * ny * nz;
    dim3 grid((unsigned)((np + 255) / 256), ncol);
    grad_dir_kernel<T><<<grid, 256, 0, st>>>(x, ldx, g, ldg, A);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("gradient launch failed: %s", cudaGetErrorString(e));
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

struct Mat3Arg {
    double m[9];
};

// Cartesian gradients of a non-orthogonal cell from the three lattice-direction gradients, in
// place: g_a <- sum_d uinv[a][d] g_d (Stress.cpp:1628-1640 and :1188-1200, uinv = uvec^-1).
template <typename T>
__global__ void cart_mix_kernel(T* __restrict__ g0, T* __restrict__ g1, T* __restrict__ g2, long long n,
                                Mat3Arg uinv) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const T a = g0[i], b = g1[i], c = g2[i];
        T r[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
            r[k] = vadd(vadd(vscale(uinv.m[3 * k], a), vscale(uinv.m[3 * k + 1], b)), vscale(uinv.m[3 * k + 2], c));
        g0[i] = r[0];
        g1[i] = r[1];
        g2[i] = r[2];
    }
}

template <typename T>
int launch_cart_mix(T* g0, T* g1, T* g2, long long n, const double* uinv, cudaStream_t st) {
    Mat3Arg m;
    for (int k = 0; k < 9; ++k) m.m[k] = uinv[k];
    cart_mix_kernel<T><<<1184, 256, 0, st>>>(g0, g1, g2, n, m);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("gradient mixing launch failed: %s", cudaGetErrorString(e));
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

__device__ __forceinline__ double re_dot(double a, double b) { return a * b; }
__device__ __forceinline__ double re_dot(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }

// Six Voigt products of every column, out[v * ncol + n] = sum_i Re(conj(g_a(i, n)) g_b(i, n)),
// (a, b) = xx, xy, xz, yy, yz, zz.  CTA = one column; each thread sums a fixed strided subset of
// the points and the block adds the partials in a fixed tree, so the result is reproducible.
template <typename T>
__global__ void __launch_bounds__(256) dot6_kernel(const T* __restrict__ g0, const T* __restrict__ g1,
                                                   const T* __restrict__ g2, long long nd, long long ld,
                                                   int ncol, double* __restrict__ out) {
    __shared__ double red[6][256];
    const int n = blockIdx.x;
    const T* a0 = g0 + (long long)n * ld;
    const T* a1 = g1 + (long long)n * ld;
    const T* a2 = g2 + (long long)n * ld;
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (long long i = threadIdx.x; i < nd; i += blockDim.x) {
        const T x = a0[i], y = a1[i], z = a2[i];
        s[0] += re_dot(x, x);
        s[1] += re_dot(x, y);
        s[2] += re_dot(x, z);
        s[3] += re_dot(y, y);
        s[4] += re_dot(y, z);
        s[5] += re_dot(z, z);
    }
#pragma unroll
    for (int v = 0; v < 6; ++v) red[v][threadIdx.x] = s[v];
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
#pragma unroll
            for (int v = 0; v < 6; ++v) red[v][threadIdx.x] += red[v][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x < 6) out[(long long)threadIdx.x * ncol + n] = red[threadIdx.x][0];
}

template <typename T>
int launch_dot6(const T* g0, const T* g1, const T* g2, long long nd, long long ld, int ncol, double* out,
                cudaStream_t st) {
    if (ncol <= 0) return LYNX_OK;
    dot6_kernel<T><<<ncol, 256, 0, st>>>(g0, g1, g2, nd, ld, ncol, out);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("gradient products launch failed: %s", cudaGetErrorString(e));
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

template int launch_cart_mix<double>(double*, double*, double*, long long, const double*, cudaStream_t);
template int launch_cart_mix<double2>(double2*, double2*, double2*, long long, const double*, cudaStream_t);
template int launch_dot6<double>(const double*, const double*, const double*, long long, long long, int, double*,
                                 cudaStream_t);
template int launch_dot6<double2>(const double2*, const double2*, const double2*, long long, long long, int, double*,
                                  cudaStream_t);

template int launch_grad_dir<double>(int, int, int, int, int, const double*, int, const double*, long long, double*,
                                     long long, int, const double*, const double*, cudaStream_t);
template int launch_grad_dir<double2>(int, int, int, int, int, const double*, int, const double2*, long long, double2*,
                                      long long, int, const double2*, const double2*, cudaStream_t);

}  // namespace lynxb
