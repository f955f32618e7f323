// Launch-shape selection and template dispatch for the pipelined Chebyshev-step kernel.
// LYNX_STENCIL_TYPES = 0: real (double, float); 1: complex (double2, float2).
#include <algorithm>
#include <cstdio>
#include <type_traits>

#include "kernels.h"
#include "lynx_common.cuh"
#include "stencil_pipe.cuh"

namespace lynxb {

namespace {

// Launch shapes: RX adjacent x points x RY rows per thread, launch-bound thread count (which
// sets the register budget).  Shape 0 is the default; for the common FD half-width kTunedR the
// other shapes are compiled too and chosen per grid by the caller's autotuner (they trade
// registers per thread, i.e. window rows, against resident warps).
template <typename T, int I> struct PipeShapeAt;
template <> struct PipeShapeAt<float, 0> { static constexpr int RX = 2, RY = 4, MAXT = 352; };
template <> struct PipeShapeAt<float, 1> { static constexpr int RX = 2, RY = 3, MAXT = 512; };
template <> struct PipeShapeAt<float, 2> { static constexpr int RX = 2, RY = 2, MAXT = 512; };
template <> struct PipeShapeAt<float, 3> { static constexpr int RX = 2, RY = 3, MAXT = 448; };
template <> struct PipeShapeAt<double, 0> { static constexpr int RX = 2, RY = 2, MAXT = 352; };
template <> struct PipeShapeAt<double, 1> { static constexpr int RX = 2, RY = 1, MAXT = 512; };
template <> struct PipeShapeAt<double, 2> { static constexpr int RX = 2, RY = 1, MAXT = 640; };
template <> struct PipeShapeAt<double, 3> { static constexpr int RX = 2, RY = 2, MAXT = 384; };
template <> struct PipeShapeAt<float2, 0> { static constexpr int RX = 1, RY = 4, MAXT = 352; };
template <> struct PipeShapeAt<double2, 0> { static constexpr int RX = 1, RY = 2, MAXT = 352; };
template <typename T> struct NumShapes { static constexpr int value = 1; };
template <> struct NumShapes<float> { static constexpr int value = 4; };
template <> struct NumShapes<double> { static constexpr int value = 4; };
constexpr int kTunedR = 6;  // FD order 12

struct ShapeRT {
    int RX, RY, MAXT;
};
template <typename T, int I>
ShapeRT shape_i() {
    using P = PipeShapeAt<T, I>;
    return {P::RX, P::RY, P::MAXT};
}
template <typename T>
ShapeRT shape_rt(int si) {
    if constexpr (NumShapes<T>::value > 1) {
        switch (si) {
            case 1: return shape_i<T, 1>();
            case 2: return shape_i<T, 2>();
            case 3: return shape_i<T, 3>();
            default: break;
        }
    }
    return shape_i<T, 0>();
}

template <typename T, int R, bool XOLD, bool PH, int SI, bool NLF = false>
void launch_pipe_ph(int ns, dim3 grid, int nthr, size_t smem, cudaStream_t st, const T* x, const T* xo, T* out,
                    const typename ScalarOf<T>::type* V, const PipeGeom& G, const PipeCoef<T>& C,
                    const PipeNL<T>& NL, int* err) {
    using P = PipeShapeAt<T, SI>;
    constexpr int RX = P::RX, RY = P::RY, MT = P::MAXT;
    auto kern = ns >= 5 ? cheb_pipe_kernel<T, R, RX, RY, XOLD, 5, PH, MT, NLF>
               : (ns == 4 ? cheb_pipe_kernel<T, R, RX, RY, XOLD, 4, PH, MT, NLF>
                          : cheb_pipe_kernel<T, R, RX, RY, XOLD, 3, PH, MT, NLF>);
    smem_cap(kern, smem);
    kern<<<grid, nthr, smem, st>>>(x, xo, out, V, G, C, NL, err);
}

// Real data with periodic boundaries needs no phase on wrapped neighbours; complex data and
// Dirichlet boundaries use the PHASED instantiation (default shape only).
template <typename T, int R, bool XOLD>
void launch_pipe(int si, int ns, bool phased, bool nlf, dim3 grid, int nthr, size_t smem, cudaStream_t st, const T* x,
                 const T* xo, T* out, const typename ScalarOf<T>::type* V, const PipeGeom& G, const PipeCoef<T>& C,
                 const PipeNL<T>& NL, int* err) {
    if (ScalarOf<T>::cplx || phased) {
        launch_pipe_ph<T, R, XOLD, true, 0>(ns, grid, nthr, smem, st, x, xo, out, V, G, C, NL, err);
        return;
    }
    if constexpr (R == kTunedR && NumShapes<T>::value > 1) {
        if (nlf) {
            switch (si) {
                case 1: launch_pipe_ph<T, R, XOLD, false, 1, true>(ns, grid, nthr, smem, st, x, xo, out, V, G, C, NL, err); return;
                case 2: launch_pipe_ph<T, R, XOLD, false, 2, true>(ns, grid, nthr, smem, st, x, xo, out, V, G, C, NL, err); return;
                case 3: launch_pipe_ph<T, R, XOLD, false, 3, true>(ns, grid, nthr, smem, st, x, xo, out, V, G, C, NL, err); return;
                default: launch_pipe_ph<T, R, XOLD, false, 0, true>(ns, grid, nthr, smem, st, x, xo, out, V, G, C, NL, err); return;
            }
        }
        switch (si) {
            case 1: launch_pipe_ph<T, R, XOLD, false, 1>(ns, grid, nthr, smem, st, x, xo, out, V, G, C, NL, err); return;
            case 2: launch_pipe_ph<T, R, XOLD, false, 2>(ns, grid, nthr, smem, st, x, xo, out, V, G, C, NL, err); return;
            case 3: launch_pipe_ph<T, R, XOLD, false, 3>(ns, grid, nthr, smem, st, x, xo, out, V, G, C, NL, err); return;
            default: break;
        }
    }
    launch_pipe_ph<T, R, XOLD, false, 0>(ns, grid, nthr, smem, st, x, xo, out, V, G, C, NL, err);
}

template <typename T>
bool phases_trivial(const T* phl, const T* phr) {
    using S = typename ScalarOf<T>::type;
    for (int k = 0; k < 3; ++k) {
        const S* l = reinterpret_cast<const S*>(&phl[k]);
        const S* r = reinterpret_cast<const S*>(&phr[k]);
        for (int c = 0; c < (int)(sizeof(T) / sizeof(S)); ++c)
            if (l[c] != (c == 0 ? S(1) : S(0)) || r[c] != (c == 0 ? S(1) : S(0))) return false;
    }
    return true;
}

}  // namespace

template <typename T>
int pipe_shape_count(int R) {
    // shapes x band splits: index = shape + NumShapes * (extra y-bands, 0 or 1)
    return (R == kTunedR && NumShapes<T>::value > 1) ? 2 * NumShapes<T>::value : 1;
}

template <typename T, typename S>
int launch_cheb_pipe(const StencilGeom& g, int nxp, const T* x, long long ldx, const T* xold, long long ldo, T* out,
                     long long ldout, const S* V, int ncol, double a, double b, double d, const T* phl, const T* phr,
                     int* err, cudaStream_t st, int shape, const PipeNLHost* nlh) {
    static_assert(std::is_same<S, typename ScalarOf<T>::type>::value, "scalar type mismatch");
    const int R = g.R;
    const bool phased = ScalarOf<T>::cplx || !phases_trivial(phl, phr);
    const bool nlf = nlh != nullptr;
    if (nlf && (R != kTunedR || phased || NumShapes<T>::value == 1)) {
        set_error("fused nonlocal term needs real data, periodic cells and FD order 12");
        return LYNX_ERR_UNSUPPORTED;
    }
    const int sidx = (shape > 0 && shape < pipe_shape_count<T>(R) && !phased) ? shape : 0;
    const int si = sidx % NumShapes<T>::value;    // compiled launch shape
    const int extra_bands = sidx / NumShapes<T>::value;  // one more y-band: more, shorter CTAs
    const ShapeRT sh = shape_rt<T>(si);
    const int RX = sh.RX, RY = sh.RY, MT = sh.MAXT;
    if (R < 1 || R > 8) {
        set_error("FD half-width %d outside the supported range 1..8", R);
        return LYNX_ERR_UNSUPPORTED;
    }
    if (g.nx < R || g.ny < R || g.nz < R) {
        set_error("grid %dx%dx%d smaller than the FD half-width %d", g.nx, g.ny, g.nz, R);
        return LYNX_ERR_UNSUPPORTED;
    }
    if (nxp < g.nx || (nxp * sizeof(S)) % 16 != 0 || (ldx * sizeof(T)) % 16 || (ldout * sizeof(T)) % 16 ||
        (xold && (ldo * sizeof(T)) % 16)) {
        set_error("pipelined stencil needs 16-byte aligned rows and columns");
        return LYNX_ERR_BAD_ARG;
    }
    if (g.nx % RX != 0) {
        set_error("pipelined stencil needs nx to be a multiple of %d", RX);
        return LYNX_ERR_UNSUPPORTED;
    }
    if (ncol <= 0) return LYNX_OK;
    const int P2 = g.nx / RX;
    if (P2 > MT - 32) {
        set_error("nx = %d too large for the pipelined stencil", g.nx);
        return LYNX_ERR_UNSUPPORTED;
    }
    // One CTA per SM: about MT - 64 consumer threads (whole x-rows per thread row), bands
    // balanced over ny.
    int TYT = std::max(1, (MT - 64 + P2 / 2) / P2);
    TYT = std::min(TYT, (MT - 32) / P2);
    TYT = std::min(TYT, (g.ny + RY - 1) / RY);
    {
        const int nb = std::min(g.ny, (g.ny + TYT * RY - 1) / (TYT * RY) + extra_bands);
        const int ty_bal = (g.ny + nb - 1) / nb;
        TYT = std::max(1, std::min(TYT, (ty_bal + RY - 1) / RY));
    }
    const int nthr = ((P2 * TYT + 31) / 32) * 32 + 32;  // consumer warps + one producer warp
    PipeGeom G;
    G.nx = g.nx;
    G.ny = g.ny;
    G.nz = g.nz;
    G.nxp = nxp;
    G.GL = 0;
    G.SP = nxp;
    G.TYT = TYT;
    G.TY = TYT * RY;
    G.P2 = P2;
    G.plane = (long long)nxp * g.ny;
    G.ld_x = ldx;
    G.ld_old = ldo;
    G.ld_out = ldout;
    const int nbands = (g.ny + G.TY - 1) / G.TY;
    const long long base = (long long)nbands * ncol;
    int nzch = (int)std::min<long long>((600 + base - 1) / base, std::max(1, g.nz / (4 * R)));
    nzch = std::max(1, nzch);
    G.zchunk = (g.nz + nzch - 1) / nzch;
    nzch = (g.nz + G.zchunk - 1) / G.zchunk;
    const bool xo = (xold != nullptr) && d != 0.0;
    const size_t own_b = (size_t)G.TY * nxp * sizeof(T);
    PipeNL<T> NL{};
    if (nlf) {
        NL.W = static_cast<const T*>(nlh->W);
        NL.ldw = nlh->ldw;
        NL.ptmap = nlh->ptmap;
        NL.mp = nlh->mp;
        NL.rowstart = nlh->rowstart;
        NL.xs_out = static_cast<T*>(nlh->xs_out);
        // largest 16-byte-rounded W range of one band-plane for this band height
        const int VWn = 16 / (int)sizeof(T);
        const std::vector<int>& rs = *nlh->rowstart_host;
        int wcap = 0;
        for (int z = 0; z < g.nz; ++z)
            for (int y0 = 0; y0 < g.ny; y0 += G.TY) {
                const int tyv = std::min(G.TY, g.ny - y0);
                const int ps = rs[(size_t)z * g.ny + y0], pe = rs[(size_t)z * g.ny + y0 + tyv];
                wcap = std::max(wcap, ((pe + VWn - 1) & ~(VWn - 1)) - (ps & ~(VWn - 1)));
            }
        NL.wcap = wcap;
    }
    const size_t stage = (size_t)pipe_stage_layout(G.TY, R, nxp, (int)sizeof(T), (int)sizeof(S), xo, nlf, NL.mp,
                                                   NL.wcap).bytes;
    // window ring (4 stages of the band's own rows) + as many tile stages (3..5) as fit
    const size_t wring = 4 * ((own_b + 127) / 128) * 128 + (nlf ? (size_t)8 * G.zchunk : 0);  // + W range table
    int ns = (int)std::min<size_t>(5, (227 * 1024 - 256 - wring) / stage);
    const size_t smem = 256 + wring + (size_t)std::max(ns, 3) * stage;
    if (smem > 227 * 1024) {
        set_error("pipelined stencil stage of %zu bytes exceeds shared memory", smem);
        return LYNX_ERR_UNSUPPORTED;
    }
    if (ncol > 65535 || nzch > 65535) {
        set_error("too many columns (%d) for one launch", ncol);
        return LYNX_ERR_UNSUPPORTED;
    }
    PipeCoef<T> C;
    for (int p = 0; p <= 8; ++p) C.cx[p] = C.cy[p] = C.cz[p] = S(0);
    for (int p = 1; p <= R; ++p) {
        C.cx[p] = (S)(-0.5 * a * g.D2x[p]);
        C.cy[p] = (S)(-0.5 * a * g.D2y[p]);
        C.cz[p] = (S)(-0.5 * a * g.D2z[p]);
    }
    centre_coef<S>(g, a, b, C.cx, C.cy, C.cz, &C.diag, &C.diag_lo);
    C.a = (S)a;
    C.d = (S)d;
    for (int k = 0; k < 3; ++k) {
        C.phl[k] = phl[k];
        C.phr[k] = phr[k];
    }
    dim3 grid(nbands, ncol, nzch);
#define LYNX_PIPE_CASE(RR)                                                                       \
    case RR:                                                                                     \
        if (xo) launch_pipe<T, RR, true>(si, ns, phased, nlf, grid, nthr, smem, st, x, xold, out, V, G, C, NL, err); \
        else launch_pipe<T, RR, false>(si, ns, phased, nlf, grid, nthr, smem, st, x, xold, out, V, G, C, NL, err);   \
        break;
    switch (R) {
        LYNX_PIPE_CASE(1)
        LYNX_PIPE_CASE(2)
        LYNX_PIPE_CASE(3)
        LYNX_PIPE_CASE(4)
        LYNX_PIPE_CASE(5)
        LYNX_PIPE_CASE(6)
        LYNX_PIPE_CASE(7)
        LYNX_PIPE_CASE(8)
    }
#undef LYNX_PIPE_CASE
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("pipelined stencil launch failed: %s", cudaGetErrorString(e));
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

#if LYNX_STENCIL_TYPES == 0
template int launch_cheb_pipe<double, double>(const StencilGeom&, int, const double*, long long, const double*,
                                              long long, double*, long long, const double*, int, double, double,
                                              double, const double*, const double*, int*, cudaStream_t, int, const PipeNLHost*);
template int launch_cheb_pipe<float, float>(const StencilGeom&, int, const float*, long long, const float*,
                                            long long, float*, long long, const float*, int, double, double, double,
                                            const float*, const float*, int*, cudaStream_t, int, const PipeNLHost*);
template int pipe_shape_count<double>(int);
template int pipe_shape_count<float>(int);
#else
template int launch_cheb_pipe<double2, double>(const StencilGeom&, int, const double2*, long long, const double2*,
                                               long long, double2*, long long, const double*, int, double, double,
                                               double, const double2*, const double2*, int*, cudaStream_t, int, const PipeNLHost*);
template int launch_cheb_pipe<float2, float>(const StencilGeom&, int, const float2*, long long, const float2*,
                                             long long, float2*, long long, const float*, int, double, double,
                                             double, const float2*, const float2*, int*, cudaStream_t, int, const PipeNLHost*);
template int pipe_shape_count<double2>(int);
template int pipe_shape_count<float2>(int);
#endif

}  // namespace lynxb
