// Effective potential on sm_100a: the rest of an SCF iteration's potential update
// (src/physics/EffectivePotential.cpp:44-177, non-spin-polarised):
//   * FD first derivatives of a scalar field (src/operators/Gradient.cpp:17-60), periodic or
//     zero (Dirichlet) ghosts per direction;
//   * GGA-PBE exchange-correlation per grid point and the divergence of the GGA flux
//     (src/xc/XCFunctional.cpp:193-273; the reference evaluates the functional with libxc's
//     XC_GGA_X_PBE + XC_GGA_C_PBE, here it is this file's own restatement of the published
//     functional, below);
//   * the vector kernels of the AAR Poisson iteration (src/solvers/PoissonSolver.cpp:43-159):
//     fused preconditioner / history / save, Richardson and Anderson updates, residual, and
//     deterministic dot products (fixed block partition, fixed-order sums).
// FP64 throughout; one field of nd = nx ny nz points, x fastest.
#include <cmath>

#include "kernels.h"
#include "lynx_common.cuh"

namespace lynxb {

namespace {

constexpr int kVThreads = 256;
constexpr int kDotBlocks = 296;  // 2 x 148 SMs: the dot-product partition (fixed, so sums are reproducible)

__device__ __forceinline__ int wrap_idx(int i, int n, bool periodic, bool* zero) {
    if (i < 0) {
        if (!periodic) *zero = true;
        return i + n;
    }
    if (i >= n) {
        if (!periodic) *zero = true;
        return i - n;
    }
    return i;
}

// d/d(direction) of x at point (i, j, k): sum_{p=1..R} D1[p] (x[+p] - x[-p]), accumulated from zero
// in increasing p (the reference's order); ghosts wrap (periodic) or read zero (Dirichlet).
__device__ __forceinline__ double fd_deriv(const double* __restrict__ x, const GradGeom& g, int dir, int i, int j,
                                           int k) {
    double val = 0.0;
    const int n = dir == 0 ? g.nx : dir == 1 ? g.ny : g.nz;
    const int c = dir == 0 ? i : dir == 1 ? j : k;
    const bool per = g.periodic[dir] != 0;
    for (int p = 1; p <= g.R; ++p) {
        bool zp = false, zm = false;
        const int cp = wrap_idx(c + p, n, per, &zp);
        const int cm = wrap_idx(c - p, n, per, &zm);
        long long ip, im;
        if (dir == 0) {
            ip = ((long long)k * g.ny + j) * g.nx + cp;
            im = ((long long)k * g.ny + j) * g.nx + cm;
        } else if (dir == 1) {
            ip = ((long long)k * g.ny + cp) * g.nx + i;
            im = ((long long)k * g.ny + cm) * g.nx + i;
        } else {
            ip = ((long long)cp * g.ny + j) * g.nx + i;
            im = ((long long)cm * g.ny + j) * g.nx + i;
        }
        const double xp = zp ? 0.0 : x[ip];
        const double xm = zm ? 0.0 : x[im];
        val += g.D1[dir][p] * (xp - xm);
    }
    return val;
}

__global__ void grad3_kernel(const double* __restrict__ x, GradGeom g, double* __restrict__ dx,
                             double* __restrict__ dy, double* __restrict__ dz) {
    const long long nd = (long long)g.nx * g.ny * g.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nd; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % g.nx);
        const int j = (int)((t / g.nx) % g.ny);
        const int k = (int)(t / ((long long)g.nx * g.ny));
        dx[t] = fd_deriv(x, g, 0, i, j, k);
        dy[t] = fd_deriv(x, g, 1, i, j, k);
        dz[t] = fd_deriv(x, g, 2, i, j, k);
    }
}

// v[t] -= d_x fx, then -= d_y fy, then -= d_z fz (the reference's three separate updates, in order).
__global__ void div_sub_kernel(double* __restrict__ v, GradGeom g, const double* __restrict__ fx,
                               const double* __restrict__ fy, const double* __restrict__ fz) {
    const long long nd = (long long)g.nx * g.ny * g.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nd; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % g.nx);
        const int j = (int)((t / g.nx) % g.ny);
        const int k = (int)(t / ((long long)g.nx * g.ny));
        double a = v[t];
        a -= fd_deriv(fx, g, 0, i, j, k);
        a -= fd_deriv(fy, g, 1, i, j, k);
        a -= fd_deriv(fz, g, 2, i, j, k);
        v[t] = a;
    }
}

// ------------------------------------------------------------------------------------------
// GGA-PBE, spin-unpolarised, as published: J. P. Perdew, K. Burke, M. Ernzerhof, Phys. Rev.
// Lett. 77, 3865 (1996), with the uniform-gas correlation of J. P. Perdew, Y. Wang, Phys. Rev.
// B 45, 13244 (1992).  Energy per particle
//   eps = eps_x^unif(rho) F_x(s) + eps_c^unif(r_s) + H(r_s, t),
//   eps_x^unif = -(3/4)(3/pi)^(1/3) rho^(1/3),  k_F = (3 pi^2 rho)^(1/3),  s^2 = sigma / (2 k_F rho)^2,
//   F_x = 1 + kappa - kappa / (1 + mu s^2 / kappa),
//   eps_c^unif = -2 A (1 + a1 r_s) ln(1 + 1 / (2 A (b1 r_s^(1/2) + b2 r_s + b3 r_s^(3/2) + b4 r_s^2))),
//   t^2 = sigma / (2 k_s rho)^2 with k_s^2 = 4 k_F / pi,
//   H = gamma ln(1 + (beta/gamma) t^2 (1 + A' t^2) / (1 + A' t^2 + A'^2 t^4)),
//   A' = (beta/gamma) / (exp(-eps_c^unif / gamma) - 1),  gamma = (1 - ln 2) / pi^2.
// Constants: kappa = 0.804, beta = 0.06672455060314922, mu = beta pi^2 / 3; PW92 parameters for
// zeta = 0 with A at the 7-digit value 0.0310907 (the "modified" PW92 that PBE correlation is
// usually paired with).  vrho = d(rho eps)/d rho and vsigma = d(rho eps)/d sigma are carried
// alongside the value as forward-mode dual numbers, exact to rounding.
// ------------------------------------------------------------------------------------------
struct Dual {
    double v, r, s;  // value, d/d rho, d/d sigma
};
__device__ __forceinline__ Dual dconst(double c) { return {c, 0.0, 0.0}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.r + b.r, a.s + b.s}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.r - b.r, a.s - b.s}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) {
    return {a.v * b.v, a.r * b.v + a.v * b.r, a.s * b.v + a.v * b.s};
}
__device__ __forceinline__ Dual operator*(double c, Dual a) { return {c * a.v, c * a.r, c * a.s}; }
__device__ __forceinline__ Dual operator+(double c, Dual a) { return {c + a.v, a.r, a.s}; }
__device__ __forceinline__ Dual operator*(Dual a, double c) { return {c * a.v, c * a.r, c * a.s}; }
__device__ __forceinline__ Dual operator-(double c, Dual a) { return {c - a.v, -a.r, -a.s}; }
__device__ __forceinline__ Dual operator/(double c, Dual a) {
    const double q = c / a.v;
    return {q, -q * a.r / a.v, -q * a.s / a.v};
}
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return {q, (a.r - q * b.r) / b.v, (a.s - q * b.s) / b.v};
}
__device__ __forceinline__ Dual dlog(Dual a) { return {log(a.v), a.r / a.v, a.s / a.v}; }
__device__ __forceinline__ Dual dexp(Dual a) {
    const double e = exp(a.v);
    return {e, e * a.r, e * a.s};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
    const double q = sqrt(a.v);
    const double h = 0.5 / q;
    return {q, h * a.r, h * a.s};
}
__device__ __forceinline__ Dual dcbrt(Dual a) {
    const double q = cbrt(a.v);
    const double h = 1.0 / (3.0 * q * q);
    return {q, h * a.r, h * a.s};
}

constexpr double kPi = 3.14159265358979323846;
constexpr double kPbeKappa = 0.804;
constexpr double kPbeBeta = 0.06672455060314922;

__device__ void pbe_point(double rho, double sigma, double* exc, double* vrho, double* vsigma) {
    const double mu = kPbeBeta * kPi * kPi / 3.0;
    const double gam = (1.0 - log(2.0)) / (kPi * kPi);
    const double cx = 0.75 * cbrt(3.0 / kPi);       // -eps_x^unif / rho^(1/3)
    const double ckf = cbrt(3.0 * kPi * kPi);       // k_F / rho^(1/3)
    const double c31 = cbrt(3.0 / (4.0 * kPi));     // r_s rho^(1/3)
    const double pwA = 0.0310907, pwa1 = 0.21370, pwb1 = 7.5957, pwb2 = 3.5876, pwb3 = 1.6382, pwb4 = 0.49294;
    const Dual r{rho, 1.0, 0.0}, s{sigma, 0.0, 1.0};
    const Dual r13 = dcbrt(r);
    const Dual kf = ckf * r13;
    const Dual rr = r * r;
    // exchange
    const Dual exu = (-cx) * r13;
    const Dual s2 = s / (4.0 * (kf * kf * rr));
    const Dual fx = (1.0 + kPbeKappa) - kPbeKappa / (1.0 + (mu / kPbeKappa) * s2);
    // correlation
    const Dual rs = c31 / r13;
    const Dual srs = dsqrt(rs);
    const Dual den = (2.0 * pwA) * (pwb1 * srs + pwb2 * rs + pwb3 * (rs * srs) + pwb4 * (rs * rs));
    const Dual ecu = (-2.0 * pwA) * ((1.0 + pwa1 * rs) * dlog(1.0 + dconst(1.0) / den));
    const Dual t2 = s * (kPi / 16.0) / (kf * rr);
    const Dual Ap = (kPbeBeta / gam) / (dexp((-1.0 / gam) * ecu) - dconst(1.0));
    const Dual At2 = Ap * t2;
    const Dual H = gam * dlog(1.0 + (kPbeBeta / gam) * (t2 * (1.0 + At2) / (1.0 + At2 + At2 * At2)));
    const Dual eps = exu * fx + ecu + H;
    const Dual F = r * eps;
    *exc = eps.v;
    *vrho = F.r;
    *vsigma = F.s;
}

// rho_xc = max(rho + rho_core, 1e-14): the density the functional sees when a core density is
// given (src/physics/EffectivePotential.cpp:127-134).
__global__ void rho_xc_kernel(const double* __restrict__ rho, const double* __restrict__ core,
                              double* __restrict__ out, long long nd) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nd; t += (long long)gridDim.x * blockDim.x) {
        const double v = rho[t] + core[t];
        out[t] = (v > 1e-14) ? v : 1e-14;
    }
}

// Per point: sigma from the gradient (lapc_T metric for non-orthogonal cells), the functional,
// and the GGA flux f = v2xc lapc_T grad(rho) written over the gradient arrays.  Points with
// rho <= 1e-14 contribute nothing (exc = vrho = v2xc = 0).
__global__ void pbe_kernel(const double* __restrict__ rho, long long nd, XcMetric m, double* __restrict__ gx,
                           double* __restrict__ gy, double* __restrict__ gz, double* __restrict__ vxc,
                           double* __restrict__ exc, double* __restrict__ v2xc) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nd; t += (long long)gridDim.x * blockDim.x) {
        const double rx = rho[t];
        const double dx = gx[t], dy = gy[t], dz = gz[t];
        double sig;
        if (m.orth) {
            sig = dx * dx + dy * dy + dz * dz;
        } else {
            sig = m.L[0] * dx * dx + m.L[4] * dy * dy + m.L[8] * dz * dz + 2.0 * m.L[1] * dx * dy +
                  2.0 * m.L[2] * dx * dz + 2.0 * m.L[5] * dy * dz;
        }
        double e = 0.0, vr = 0.0, vs = 0.0;
        if (rx > 1e-14) pbe_point(rx, sig, &e, &vr, &vs);
        const double w = 2.0 * vs;
        exc[t] = e;
        vxc[t] = vr;
        if (v2xc) v2xc[t] = w;
        if (m.orth) {
            gx[t] = dx * w;
            gy[t] = dy * w;
            gz[t] = dz * w;
        } else {
            gx[t] = (m.L[0] * dx + m.L[1] * dy + m.L[2] * dz) * w;
            gy[t] = (m.L[3] * dx + m.L[4] * dy + m.L[5] * dz) * w;
            gz[t] = (m.L[6] * dx + m.L[7] * dy + m.L[8] * dz) * w;
        }
    }
}

// ------------------------------------------------------------------------------------------
// AAR vector kernels.
// ------------------------------------------------------------------------------------------
// f = w r; with col >= 0 the history column col: X = x - x_old, F = f - f_old; then x_old = x,
// f_old = f (src/solvers/PoissonSolver.cpp:103-115 in one pass).
__global__ void aar_pre_kernel(const double* __restrict__ r, const double* __restrict__ x, double* __restrict__ x_old,
                               double* __restrict__ f, double* __restrict__ f_old, double* __restrict__ X,
                               double* __restrict__ F, double w, long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const double fi = w * r[t];
        const double xi = x[t];
        if (X) {
            X[t] = xi - x_old[t];
            F[t] = fi - f_old[t];
        }
        x_old[t] = xi;
        f_old[t] = fi;
        f[t] = fi;
    }
}

// x = x_old + c f - sum_j g[j] (X_j + c F_j)   (Richardson: cols = 0, c = omega)
__global__ void aar_update_kernel(double* __restrict__ x, const double* __restrict__ x_old, const double* __restrict__ f,
                                  const double* __restrict__ X, const double* __restrict__ F, AarGamma g, double c,
                                  long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        double v = x_old[t] + c * f[t];
        for (int j = 0; j < g.cols; ++j) v -= g.g[j] * (X[(long long)j * n + t] + c * F[(long long)j * n + t]);
        x[t] = v;
    }
}

__global__ void sub_kernel(const double* __restrict__ b, const double* __restrict__ a, double* __restrict__ r,
                           long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        r[t] = b[t] - a[t];
}

// Partial sums of up to kMaxDots dot products u_k . v_k over a fixed partition of [0, n):
// part[k * gridDim.x + block].  Block sums in a fixed shared-memory tree.
__global__ void dots_partial_kernel(DotList L, long long n, double* __restrict__ part) {
    __shared__ double sh[kVThreads];
    const long long per = (n + gridDim.x - 1) / gridDim.x;
    const long long lo = blockIdx.x * per;
    const long long hi = min(n, lo + per);
    for (int k = 0; k < L.count; ++k) {
        double a = 0.0;
        for (long long t = lo + threadIdx.x; t < hi; t += blockDim.x) a += L.u[k][t] * L.v[k][t];
        sh[threadIdx.x] = a;
        __syncthreads();
        for (int h = blockDim.x / 2; h > 0; h >>= 1) {
            if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(long long)k * gridDim.x + blockIdx.x] = sh[0];
        __syncthreads();
    }
}

// out[k] = sum over blocks of part[k][*], in a fixed tree (one CTA per dot).
__global__ void dots_final_kernel(const double* __restrict__ part, int nblk, double* __restrict__ out) {
    __shared__ double sh[kVThreads];
    double a = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) a += part[(long long)blockIdx.x * nblk + b];
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

// out = sa a (+ sa b) - s   (b may be null)
__global__ void add_shift_kernel(const double* __restrict__ a, const double* __restrict__ b, double s, double sa,
                                 double* __restrict__ out, long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        double v = sa * a[t];
        if (b) v += sa * b[t];
        out[t] = v - s;
    }
}

// z[i] *= s[i] * scale over the half-spectrum of a real 3-D FFT (the periodic Poisson solve).
__global__ void spec_scale_kernel(double2* __restrict__ z, const double* __restrict__ s, double scale, long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const double f = s[t] * scale;
        z[t] = make_double2(z[t].x * f, z[t].y * f);
    }
}

// s[i] = 1 / Re(g_hat[i]) (0 for the mean mode i = 0 and for modes whose symbol vanishes).
__global__ void inv_symbol_kernel(const double2* __restrict__ g, double* __restrict__ s, long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const double v = g[t].x;
        s[t] = (t == 0 || fabs(v) < 1e-300) ? 0.0 : 1.0 / v;
    }
}

int grid_for(long long n) {
    long long b = (n + kVThreads - 1) / kVThreads;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b < 1 ? 1 : b);
}

int launch_ok(const char* what) {
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s launch failed: %s", what, cudaGetErrorString(e));
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

}  // namespace

int launch_grad3(const double* x, const GradGeom& g, double* dx, double* dy, double* dz, cudaStream_t st) {
    const long long nd = (long long)g.nx * g.ny * g.nz;
    grad3_kernel<<<grid_for(nd), kVThreads, 0, st>>>(x, g, dx, dy, dz);
    return launch_ok("gradient");
}

int launch_div_sub(double* v, const GradGeom& g, const double* fx, const double* fy, const double* fz,
                   cudaStream_t st) {
    const long long nd = (long long)g.nx * g.ny * g.nz;
    div_sub_kernel<<<grid_for(nd), kVThreads, 0, st>>>(v, g, fx, fy, fz);
    return launch_ok("GGA divergence");
}

int launch_rho_xc(const double* rho, const double* core, double* out, long long nd, cudaStream_t st) {
    rho_xc_kernel<<<grid_for(nd), kVThreads, 0, st>>>(rho, core, out, nd);
    return launch_ok("core density");
}

int launch_pbe(const double* rho, long long nd, const XcMetric& m, double* gx, double* gy, double* gz, double* vxc,
               double* exc, double* v2xc, cudaStream_t st) {
    pbe_kernel<<<grid_for(nd), kVThreads, 0, st>>>(rho, nd, m, gx, gy, gz, vxc, exc, v2xc);
    return launch_ok("GGA-PBE");
}

int launch_aar_pre(const double* r, const double* x, double* x_old, double* f, double* f_old, double* X, double* F,
                   double w, long long n, cudaStream_t st) {
    aar_pre_kernel<<<grid_for(n), kVThreads, 0, st>>>(r, x, x_old, f, f_old, X, F, w, n);
    return launch_ok("AAR preconditioner");
}

int launch_aar_update(double* x, const double* x_old, const double* f, const double* X, const double* F,
                      const AarGamma& g, double c, long long n, cudaStream_t st) {
    aar_update_kernel<<<grid_for(n), kVThreads, 0, st>>>(x, x_old, f, X, F, g, c, n);
    return launch_ok("AAR update");
}

int launch_sub(const double* b, const double* a, double* r, long long n, cudaStream_t st) {
    sub_kernel<<<grid_for(n), kVThreads, 0, st>>>(b, a, r, n);
    return launch_ok("residual");
}

int launch_add_shift(const double* a, const double* b, double s, double sa, double* out, long long n,
                     cudaStream_t st) {
    add_shift_kernel<<<grid_for(n), kVThreads, 0, st>>>(a, b, s, sa, out, n);
    return launch_ok("shift");
}

int launch_spec_scale(double2* z, const double* s, double scale, long long n, cudaStream_t st) {
    spec_scale_kernel<<<grid_for(n), kVThreads, 0, st>>>(z, s, scale, n);
    return launch_ok("spectral scale");
}

int launch_inv_symbol(const double2* g, double* s, long long n, cudaStream_t st) {
    inv_symbol_kernel<<<grid_for(n), kVThreads, 0, st>>>(g, s, n);
    return launch_ok("Poisson symbol");
}

size_t dots_work_bytes() { return sizeof(double) * ((size_t)kMaxDots * kDotBlocks + kMaxDots); }

int launch_dots(const DotList& L, long long n, void* work, double* host_out, cudaStream_t st) {
    if (L.count <= 0 || L.count > kMaxDots) {
        set_error("internal error: %d dot products (at most %d)", L.count, kMaxDots);
        return LYNX_ERR_BAD_ARG;
    }
    double* part = static_cast<double*>(work);
    double* out = part + (size_t)kMaxDots * kDotBlocks;
    dots_partial_kernel<<<kDotBlocks, kVThreads, 0, st>>>(L, n, part);
    LYNX_TRY(launch_ok("dot products"));
    dots_final_kernel<<<L.count, kVThreads, 0, st>>>(part, kDotBlocks, out);
    LYNX_TRY(launch_ok("dot products"));
    LYNX_CUDA_TRY(cudaMemcpyAsync(host_out, out, sizeof(double) * L.count, cudaMemcpyDeviceToHost, st));
    LYNX_CUDA_TRY(cudaStreamSynchronize(st));
    return LYNX_OK;
}

}  // namespace lynxb
