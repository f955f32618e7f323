// Nonlocal (Kleinman-Bylander) projector apply, Hpsi += sum_a chi_a Gamma_a dV chi_a^T psi,
// as two deterministic kernels (src/operators/NonlocalProjector.cpp:121-227 real,
// :229-347 k-point; the reference GPU version uses atomicAdd in both halves,
// src/operators/NonlocalProjector.cu:110-164,227-268).
//
//   gather : one CTA per (physical atom, block of NB columns) reduces all images
//            of the atom in a fixed order:
//              alpha[p][n] = Gamma_p * dV * sum_img e^{-i k.R_img} sum_g chi_img[g,p] psi[gpos[g], n]
//            The sum runs in FP64 for FP32 data as well.
//   scatter: one thread per (distinct grid point in the union of spheres, NB columns)
//            pulls every (image, local point) entry that lands on its grid point
//            (CSR built on the host), so no two threads write the same element:
//              out[g, n] += scale * sum_entries e^{+i k.R_img} sum_p chi_img[l,p] alpha[p][n]
// alpha is stored projector-major with a padded column stride (ncolp, a multiple
// of NB) so that the inner loops need no column guards.
#pragma once
#include <cuda_runtime.h>
#include "stencil.cuh"

namespace lynxb {

struct NLView {
    int n_atom, n_img, n_pts;
    const int* atom_img_ptr;   // n_atom+1: CSR of images per atom
    const int* atom_img_list;  // n_img
    const int* atom_nproj;     // n_atom
    const int* atom_poff;      // n_atom+1: projector offsets
    const double* gamma;       // total projectors
    const int* img_atom;       // n_img
    const int* img_ndc;        // n_img
    const long long* img_goff;     // n_img: offset into gpos / entry-local indices
    const long long* img_chi_off;  // n_img: offset into chi
    const double* img_phase;   // 2*n_img: e^{-i k.R_img} (re, im)
    const int* gpos;           // sum ndc
    const void* chi;           // sum ndc*nproj, double or float
    const int* pt_grid;        // n_pts: grid index of each distinct point
    const int* pt_ptr;         // n_pts+1
    const int* ent_img;        // sum ndc
    const int* ent_loc;        // sum ndc
};

template <typename T> struct AccOf;
template <> struct AccOf<double> { using type = double; };
template <> struct AccOf<float> { using type = double; };
template <> struct AccOf<double2> { using type = double2; };
template <> struct AccOf<float2> { using type = double2; };

__device__ __forceinline__ double to_acc(double v) { return v; }
__device__ __forceinline__ double to_acc(float v) { return (double)v; }
__device__ __forceinline__ double2 to_acc(double2 v) { return v; }
__device__ __forceinline__ double2 to_acc(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ void from_acc(double& d, double v) { d = v; }
__device__ __forceinline__ void from_acc(float& d, double v) { d = (float)v; }
__device__ __forceinline__ void from_acc(double2& d, double2 v) { d = v; }
__device__ __forceinline__ void from_acc(float2& d, double2 v) { d = make_float2((float)v.x, (float)v.y); }
__device__ __forceinline__ double acc_phase(double v, double, double) { return v; }
__device__ __forceinline__ double2 acc_phase(double2 v, double re, double im) {
    return make_double2(v.x * re - v.y * im, v.x * im + v.y * re);
}

constexpr int kGatherTile = 64;  // grid points per shared-memory tile

template <typename T, int NB>
__global__ void __launch_bounds__(1024)
    nl_gather_kernel(const T* __restrict__ x, long long ld, int ncol, int ncolp, NLView tab,
                     T* __restrict__ alpha, double dV) {
    using S = typename ScalarOf<T>::type;
    using Acc = typename AccOf<T>::type;
    constexpr int G = kGatherTile;
    constexpr int GP = G + 1;  // padded row: avoids bank conflicts between columns
    extern __shared__ __align__(16) unsigned char smraw[];
    T* sx = reinterpret_cast<T*>(smraw);                       // NB x GP
    S* schi = reinterpret_cast<S*>(smraw + sizeof(T) * NB * GP);  // np x GP
    const S* chi = reinterpret_cast<const S*>(tab.chi);

    const int a = blockIdx.x;
    const int n0 = blockIdx.y * NB;
    const int np = tab.atom_nproj[a];
    const int poff = tab.atom_poff[a];
    const int nout = np * NB;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int jp = tid / NB, nn = tid - (tid / NB) * NB;
    Acc acc = to_acc(vzero(T()));
    for (int ii = tab.atom_img_ptr[a]; ii < tab.atom_img_ptr[a + 1]; ++ii) {
        const int im = tab.atom_img_list[ii];
        const int ndc = tab.img_ndc[im];
        const int* gp = tab.gpos + tab.img_goff[im];
        const S* ch = chi + tab.img_chi_off[im];
        Acc part = to_acc(vzero(T()));
        for (int g0 = 0; g0 < ndc; g0 += G) {
            const int gl = min(G, ndc - g0);
            __syncthreads();
            for (int e = tid; e < G * NB; e += nthr) {
                const int g = e % G, c = e / G;
                T v = vzero(T());
                if (g < gl && n0 + c < ncol) v = x[(long long)gp[g0 + g] + (long long)(n0 + c) * ld];
                sx[c * GP + g] = v;
            }
            for (int e = tid; e < G * np; e += nthr) {
                const int g = e % G, j = e / G;
                schi[j * GP + g] = (g < gl) ? ch[(long long)j * ndc + g0 + g] : S(0);
            }
            __syncthreads();
            if (tid < nout) {
                const S* cr = schi + jp * GP;
                const T* xr = sx + nn * GP;
                for (int g = 0; g < gl; ++g) part = fmac(part, (double)cr[g], to_acc(xr[g]));
            }
        }
        acc = vadd(acc, acc_phase(part, tab.img_phase[2 * im], tab.img_phase[2 * im + 1]));
    }
    if (tid < nout) {
        T out;
        from_acc(out, vscale(tab.gamma[poff + jp] * dV, acc));
        alpha[(long long)(poff + jp) * ncolp + n0 + nn] = out;
    }
}

template <typename T, int NB>
__global__ void __launch_bounds__(128)
    nl_scatter_kernel(T* __restrict__ out, long long ld, int ncol, int ncolp, NLView tab,
                      const T* __restrict__ alpha, typename ScalarOf<T>::type scale) {
    using S = typename ScalarOf<T>::type;
    const S* chi = reinterpret_cast<const S*>(tab.chi);
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= tab.n_pts) return;
    const int n0 = blockIdx.y * NB;
    T acc[NB];
#pragma unroll
    for (int k = 0; k < NB; ++k) acc[k] = vzero(T());
    for (int e = tab.pt_ptr[u]; e < tab.pt_ptr[u + 1]; ++e) {
        const int im = tab.ent_img[e];
        const int l = tab.ent_loc[e];
        const int a = tab.img_atom[im];
        const int np = tab.atom_nproj[a];
        const int poff = tab.atom_poff[a];
        const int ndc = tab.img_ndc[im];
        const S* ch = chi + tab.img_chi_off[im] + l;
        T tmp[NB];
#pragma unroll
        for (int k = 0; k < NB; ++k) tmp[k] = vzero(T());
        for (int j = 0; j < np; ++j) {
            const S c = ch[(long long)j * ndc];
            const T* al = alpha + (long long)(poff + j) * ncolp + n0;
#pragma unroll
            for (int k = 0; k < NB; ++k) tmp[k] = fmac(tmp[k], c, al[k]);
        }
        if constexpr (ScalarOf<T>::cplx) {
            // conj of the gather phase: e^{+i k.R_img}
            T ph;
            ph.x = (S)tab.img_phase[2 * im];
            ph.y = -(S)tab.img_phase[2 * im + 1];
#pragma unroll
            for (int k = 0; k < NB; ++k) acc[k] = vadd(acc[k], pmul(tmp[k], ph));
        } else {
#pragma unroll
            for (int k = 0; k < NB; ++k) acc[k] = vadd(acc[k], tmp[k]);
        }
    }
    T* o = out + tab.pt_grid[u];
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        if (n0 + k < ncol) {
            T* p = o + (long long)(n0 + k) * ld;
            *p = fmac(*p, scale, acc[k]);
        }
    }
}

}  // namespace lynxb
