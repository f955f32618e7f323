// Host-side launch interfaces of the lynx_b200 kernels (implemented in the .cu files).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

namespace lynxb {

constexpr int kMaxR1 = 9;  // FD half-width bound + 1 (coefficient arrays 0..R)

// Geometry + FD coefficients of one cell for the fused stencil kernel.
struct StencilGeom {
    int nx, ny, nz;
    int R;               // FD half-width
    const double* D2x;   // FDn+1 scaled second-derivative coefficients (host)
    const double* D2y;
    const double* D2z;
};

// Mixed-derivative coefficients of a non-orthogonal cell (host arrays of R+1 values).
struct NonOrthGeom {
    int nx, ny, nz, R;
    const double* D1y;
    const double* D1z;
    const double* D2xy;
    const double* D2xz;
    const double* D2yz;
};
// out += a * (-1/2) * (mixed-derivative part of Lap x); gy, gz: scratch blocks like x (column
// stride ldg).  nonorth.cu.
template <typename T>
int launch_nonorth_terms(const NonOrthGeom& g, int nxp, const T* x, long long ldx, T* gy, T* gz, long long ldg, T* out,
                         long long ldout, int ncol, double a, const T* phl, const T* phr, cudaStream_t st);

// out = a*(-0.5*Lap x + V.*x) + b*x + d*xold over ncol columns (xold may be null when d == 0).
// phl/phr: per-direction ghost multipliers (3 values of T each).
template <typename T, typename S>
int launch_cheb_step(const StencilGeom& g, const T* x, long long ldx, const T* xold, long long ldo, T* out,
                     long long ldout, const S* V, int ncol, double a, double b, double d, const T* phl,
                     const T* phr, cudaStream_t st);

// Centre coefficient of a Chebyshev step, -0.5 a (D2x[0] + D2y[0] + D2z[0]) + b, for neighbour
// coefficients c[p] = -0.5 a D2[p] stored in precision S, returned as a (hi, lo) pair in S.
// FP32 (S = float): the centre is moved by the neighbours' rounding, -2 sum (c32 - c64), so the
// FP32 operator keeps the FP64 row sum (a constant keeps its exact kinetic energy), and it is
// carried as two floats.  A single float of ~40 Ha is off by up to 1.3e-6 Ha, and so would be
// every Ritz value of the mixed pass, shifted uniformly.  FP64: hi = the centre, lo = 0.
template <typename S>
void centre_coef(const StencilGeom& g, double a, double b, const S* cx, const S* cy, const S* cz, S* hi, S* lo) {
    double c = -0.5 * a * (g.D2x[0] + g.D2y[0] + g.D2z[0]) + b;
    if (sizeof(S) == sizeof(float)) {
        for (int p = 1; p <= g.R; ++p)
            c -= 2.0 * (((double)cx[p] + 0.5 * a * g.D2x[p]) + ((double)cy[p] + 0.5 * a * g.D2y[p]) +
                        ((double)cz[p] + 0.5 * a * g.D2z[p]));
    }
    *hi = (S)c;
    *lo = (S)(c - (double)*hi);
}

// Padded row length used by the pipelined stencil: rows and Veff rows must be 16-byte multiples.
inline int pipe_row_elems(int nx, size_t scalar_size) {
    const int q = (int)(16 / scalar_size);
    return ((nx + q - 1) / q) * q;
}

// Fused nonlocal term for the pipelined stencil: out += a * W[ptmap[point]] at sphere points
// (W: compact (chi alpha) values, column stride ldw; ptmap row pitch mp; rowstart and its host
// copy: first compact point number of every grid row (z * ny + y), nz * ny + 1 entries).
struct PipeNLHost {
    const void* W;
    long long ldw;
    const int* ptmap;
    int mp;
    const int* rowstart;
    const std::vector<int>* rowstart_host;
    void* xs_out;  // optional compact copy of out at the sphere points (column stride ldw)
};

// Pipelined stencil on 16-byte aligned, row-padded (nxp) blocks; V padded the same way.
// err: device int set to 1 if a bounded shared-memory wait gives up.
template <typename T, typename S>
int launch_cheb_pipe(const StencilGeom& g, int nxp, const T* x, long long ldx, const T* xold, long long ldo, T* out,
                     long long ldout, const S* V, int ncol, double a, double b, double d, const T* phl, const T* phr,
                     int* err, cudaStream_t st, int shape = 0, const struct PipeNLHost* nlh = nullptr);
// Number of launch shapes for FD half-width R: compiled shapes x two y-band splits (shape
// indices 0 .. count-1; any shape gives bitwise the same result, they differ in speed only).
template <typename T>
int pipe_shape_count(int R);

// Rayleigh-Ritz Gram products Ms = dV Y^T Y (upper triangle), Hs = dV Y^T HY of FP32 blocks
// (rows x n, column stride ld) on the tensor cores: exact int8-slice products, FP64 result,
// Ms/Hs n x n column-major.  work: gram_plan(rows, n).work_bytes, 256-byte aligned.
// nonfinite (device int, may be null) is set to 1 when Y or HY holds a NaN or Inf.
struct GramPlan {
    long long ldk;      // padded K (rows) of the slice arrays
    int npad;           // N rounded up to the 128-state tile
    int nsplit, kper;   // K chunks and 128-row K steps per chunk
    size_t slice_bytes, exp_bytes, ws_bytes, work_bytes;
};
GramPlan gram_plan(long long rows, int n);
int launch_gram_i8(const float* Y, const float* HY, long long ld, long long rows, int n, double dV,
                   const GramPlan& p, void* work, size_t work_bytes, double* Ms, double* Hs, int* err,
                   int* nonfinite, cudaStream_t st);

// Subspace rotation psi = Y W on the tensor cores (exact int8 slices, FP64 output written into
// an unpadded layout with column stride ldp); gram_tc.cu.  launch_colexp must run on the
// overlap Ms (before its Cholesky factorisation) to fix the per-state scaling.
struct RotPlan {
    long long ldk;  // row stride (bytes) of the slice arrays, >= N
    size_t a_bytes, b_bytes, erow_bytes, col_bytes, work_bytes, smem_rows;
};
RotPlan rot_plan(long long rows, int n);
bool rot_supported(int n);
int launch_colexp(const double* Ms, int n, void* work, const RotPlan& p, long long rows, cudaStream_t st);
// Electron density from the rotation's epilogue: rho[r] (+)= sum_j w[j] psi[r][j]^2 over the
// npts unpadded grid points, with the per-column-tile partials in part (ceil(n / 128) * npts
// doubles) reduced in tile order.
struct RotDensity {
    const double* w;  // [n] weights (device)
    double* part;
    double* rho;      // [npts] (device)
    long long npts;
    bool accumulate;
};
int launch_rot_i8(const float* Y, long long ldy, long long rows, int nx, int nxp, const double* W, int n,
                  const RotPlan& p, void* work, size_t work_bytes, double* psi, long long ldp, int* err,
                  cudaStream_t st, const RotDensity* dens = nullptr);
// rho[i] (+)= sum_n w[n] |psi[n * ld + i]|^2 over nd points (T = double or double2; w device).
template <typename T>
int launch_density(const T* psi, long long ld, long long nd, int ncol, const double* w, double* rho, bool accumulate,
                   cudaStream_t st);

// Effective potential (veff.cu), FP64 fields of nx ny nz points, x fastest.
struct GradGeom {
    int nx, ny, nz, R;
    int periodic[3];          // per direction: 1 periodic ghosts, 0 zero (Dirichlet) ghosts
    double D1[3][kMaxR1];     // first-derivative weights / spacing, index 1..R
};
struct XcMetric {
    int orth;
    double L[9];  // lapc_T, row-major (non-orthogonal cells)
};
constexpr int kAarMaxHist = 16;
struct AarGamma {
    int cols;
    double g[kAarMaxHist];
};
constexpr int kMaxDots = 48;
struct DotList {
    int count;
    const double* u[kMaxDots];
    const double* v[kMaxDots];
};
int launch_grad3(const double* x, const GradGeom& g, double* dx, double* dy, double* dz, cudaStream_t st);
int launch_div_sub(double* v, const GradGeom& g, const double* fx, const double* fy, const double* fz,
                   cudaStream_t st);
int launch_rho_xc(const double* rho, const double* core, double* out, long long nd, cudaStream_t st);
// GGA-PBE per point; on return gx, gy, gz hold the GGA flux v2xc lapc_T grad(rho).
int launch_pbe(const double* rho, long long nd, const XcMetric& m, double* gx, double* gy, double* gz, double* vxc,
               double* exc, double* v2xc, cudaStream_t st);
int launch_aar_pre(const double* r, const double* x, double* x_old, double* f, double* f_old, double* X, double* F,
                   double w, long long n, cudaStream_t st);
int launch_aar_update(double* x, const double* x_old, const double* f, const double* X, const double* F,
                      const AarGamma& g, double c, long long n, cudaStream_t st);
int launch_sub(const double* b, const double* a, double* r, long long n, cudaStream_t st);
// out = sa a (+ sa b) - s  (b may be null)
int launch_add_shift(const double* a, const double* b, double s, double sa, double* out, long long n,
                     cudaStream_t st);
// Periodic Poisson by FFT: z *= s * scale (half-spectrum), s = 1 / Re(FFT of the operator's
// impulse response) with the mean mode set to zero.
int launch_spec_scale(double2* z, const double* s, double scale, long long n, cudaStream_t st);
int launch_inv_symbol(const double2* g, double* s, long long n, cudaStream_t st);
size_t dots_work_bytes();
// Dot products u_k . v_k (deterministic order), copied to host_out; synchronises the stream.
int launch_dots(const DotList& L, long long n, void* work, double* host_out, cudaStream_t st);

// Launches issued by the library (diagnostic counter, incremented by every launcher).
void count_launch(int n = 1);

}  // namespace lynxb

namespace lynxb {

// Device copy of the nonlocal projector tables (see nonlocal.cuh for the layout).
constexpr int kNLMaxColors = 16;  // colour classes the register-tiled scatter accepts
constexpr int kNLTilePts = 64;    // points per tile of the register-tiled nonlocal kernels

struct NLDev {
    int n_atom = 0, n_img = 0, n_pts = 0, max_np = 0, total_proj = 0;
    // Images in colour classes with pairwise disjoint grid points (n_colors = 0: not coloured,
    // the pull-style scatter is used); class k is color_img[color_off[k] .. color_off[k+1]).
    int n_colors = 0;
    int color_off[kNLMaxColors + 1] = {};
    int* color_img = nullptr;
    // (image, first point) of every 64-point tile, colour class k at color_toff[k] .. [k+1]
    int color_toff[kNLMaxColors + 1] = {};
    int2* color_tiles = nullptr;
    // Compact per-point form (only when no grid point lies in two spheres): the distinct
    // points numbered in grid order, ent_pt[entry] = point number of every (image, point) entry.
    bool compact = false;
    int* ent_pt = nullptr;
    int2* pt_meta = nullptr;     // [n_pts] (first projector row, projector count) of the point's atom
    double* chi_pt64 = nullptr;  // [max_np][n_pts] projector values in point order
    float* chi_pt32 = nullptr;
    // Tiles of kExpTilePts consecutive points for the expansion kernel: the distinct atoms of
    // tile t in order of first appearance, exp_tile_atoms[t * exp_amax + slot] (-1 past the
    // tile's count), and every point's slot in its tile.
    int exp_amax = 0;
    int* exp_tile_atoms = nullptr;
    unsigned char* pt_slot = nullptr;
    int* atom_img_ptr = nullptr;
    int* atom_img_list = nullptr;
    int* atom_nproj = nullptr;
    int* atom_poff = nullptr;
    double* gamma = nullptr;
    int* img_atom = nullptr;
    int* img_ndc = nullptr;
    long long* img_goff = nullptr;
    long long* img_chi_off = nullptr;
    double* img_phase = nullptr;
    int* gpos = nullptr;
    double* chi64 = nullptr;
    float* chi32 = nullptr;
    int* pt_grid = nullptr;
    int* pt_ptr = nullptr;
    int* ent_img = nullptr;
    int* ent_loc = nullptr;
};

// Column block widths of the nonlocal kernels; alpha rows are padded to a multiple of kNLColBlock.
constexpr int kNLColBlock = 32;
// Points per tile of the compact expansion kernel (128 threads x 4 consecutive points).
constexpr int kExpTilePts = 512;

template <typename T>
int launch_nl_gather(const NLDev& nl, const T* x, long long ld, int ncol, T* alpha, int ncolp, double dV,
                     cudaStream_t st);
template <typename T, typename S>
int launch_nl_scatter(const NLDev& nl, T* out, long long ld, int ncol, const T* alpha, int ncolp, S scale,
                      cudaStream_t st);
// Nonlocal force of one direction and per-atom energy from projections without Gamma (alpha of
// psi, beta of its derivative), occupations occ (device): see nonlocal.cuh.
template <typename T>
int launch_nl_force_reduce(const NLDev& nl, const T* alpha, const T* beta, int ncolp, int ncol, const double* occ,
                           double spn, double efac, int dim, double* force, double* ea, cudaStream_t st);
// First derivative along lattice direction dir (D1: R+1 host coefficients); nonorth.cu.
template <typename T>
int launch_grad_dir(int nx, int ny, int nz, int nxp, int R, const double* D1, int dir, const T* x, long long ldx,
                    T* g, long long ldg, int ncol, const T* phl, const T* phr, cudaStream_t st);
// Stress helpers (nonorth.cu): in-place Cartesian mixing of three lattice-direction gradient
// blocks of n elements (uinv: 3x3 row-major uvec^-1), and the six Voigt products per column.
template <typename T>
int launch_cart_mix(T* g0, T* g1, T* g2, long long n, const double* uinv, cudaStream_t st);
template <typename T>
int launch_dot6(const T* g0, const T* g1, const T* g2, long long nd, long long ld, int ncol, double* out,
                cudaStream_t st);
// W[col * ldw + point] = (chi alpha)(point, col) on the compact point numbering (nl.compact).
template <typename T>
int launch_nl_expand(const NLDev& nl, T* W, long long ldw, int ncol, const T* alpha, int ncolp, cudaStream_t st);

}  // namespace lynxb
