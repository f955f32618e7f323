// Nonlocal (Kleinman-Bylander) projector apply, Hpsi += sum_a chi_a Gamma_a dV chi_a^T psi,
// as two deterministic kernels (src/operators/NonlocalProjector.cpp:121-227 real,
// :229-347 k-point; the reference GPU version uses atomicAdd in both halves,
// src/operators/NonlocalProjector.cu:110-164,227-268).
//
//   gather : one CTA per (physical atom, block of NB columns) reduces all images
//            of the atom in a fixed order:
//              alpha[p][n] = Gamma_p * dV * sum_img e^{-i k.R_img} sum_g chi_img[g,p] psi[gpos[g], n]
//            accumulated in the precision of the data (FP64 or FP32).
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

__device__ __forceinline__ double acc_phase(double v, double, double) { return v; }
__device__ __forceinline__ double2 acc_phase(double2 v, double re, double im) {
    return make_double2(v.x * re - v.y * im, v.x * im + v.y * re);
}

constexpr int kGatherTile = 64;  // grid points per shared-memory tile

// Accumulation type of the gather: FP64 for FP64 data, the data's own precision for FP32
// data (a sum over one atom's sphere, ~10^3 terms).
template <typename T> struct GAccOf { using type = T; };
template <> struct GAccOf<double> { using type = double; };
__device__ __forceinline__ float2 acc_phase(float2 v, double re, double im) {
    return make_float2((float)(v.x * re - v.y * im), (float)(v.x * im + v.y * re));
}
__device__ __forceinline__ float acc_phase(float v, double, double) { return v; }

// gather: CTA = (atom, NB columns), 256 threads; thread = (column n, projector group jq),
// projectors jq, jq+8, jq+16, ... (up to PJ of them).  The gathered x tile is staged in
// shared memory with lanes along the grid points (coalesced loads).
template <typename T, int NB, int PJ>
__global__ void __launch_bounds__(256)
    nl_gather_kernel(const T* __restrict__ x, long long ld, int ncol, int ncolp, NLView tab,
                     T* __restrict__ alpha, double dV) {
    using S = typename ScalarOf<T>::type;
    using A = typename GAccOf<T>::type;
    constexpr int G = kGatherTile;
    constexpr int NBP = NB + 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* xs = reinterpret_cast<T*>(smraw);                          // G x NBP
    S* cs = reinterpret_cast<S*>(smraw + sizeof(T) * G * NBP);    // G x np
    const S* chi = reinterpret_cast<const S*>(tab.chi);
    const int a = blockIdx.x;
    const int n0 = blockIdx.y * NB;
    const int np = tab.atom_nproj[a];
    const int poff = tab.atom_poff[a];
    const int tid = threadIdx.x;
    const int n = tid % NB;
    const int jq = tid / NB;
    constexpr int JG = 256 / NB;  // projector groups
    A acc[PJ];
#pragma unroll
    for (int m = 0; m < PJ; ++m) acc[m] = vzero(A());
    for (int ii = tab.atom_img_ptr[a]; ii < tab.atom_img_ptr[a + 1]; ++ii) {
        const int im = tab.atom_img_list[ii];
        const int ndc = tab.img_ndc[im];
        const int* gp = tab.gpos + tab.img_goff[im];
        const S* ch = chi + tab.img_chi_off[im];
        A part[PJ];
#pragma unroll
        for (int m = 0; m < PJ; ++m) part[m] = vzero(A());
        for (int g0 = 0; g0 < ndc; g0 += G) {
            const int gl = min(G, ndc - g0);
            __syncthreads();
            for (int e = tid; e < G * NB; e += 256) {
                const int g = e % G, c = e / G;
                T v = vzero(T());
                if (g < gl && n0 + c < ncol) v = x[(long long)gp[g0 + g] + (long long)(n0 + c) * ld];
                xs[g * NBP + c] = v;
            }
            for (int e = tid; e < G * np; e += 256) {
                const int g = e % G, j = e / G;
                cs[g * np + j] = (g < gl) ? ch[(long long)j * ndc + g0 + g] : S(0);
            }
            __syncthreads();
            for (int g = 0; g < gl; ++g) {
                const T xv = xs[g * NBP + n];
#pragma unroll
                for (int m = 0; m < PJ; ++m) {
                    const int j = jq + m * JG;
                    if (j < np) part[m] = fmac(part[m], (S)cs[g * np + j], xv);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < PJ; ++m)
            acc[m] = vadd(acc[m], acc_phase(part[m], tab.img_phase[2 * im], tab.img_phase[2 * im + 1]));
    }
#pragma unroll
    for (int m = 0; m < PJ; ++m) {
        const int j = jq + m * JG;
        if (j < np) alpha[(long long)(poff + j) * ncolp + n0 + n] = vscale((S)(tab.gamma[poff + j] * dV), acc[m]);
    }
}

template <typename T, int V> struct VecN;
template <> struct VecN<float, 4> { using type = float4; };
template <> struct VecN<double, 2> { using type = double2; };
template <> struct VecN<float2, 2> { using type = float4; };
template <> struct VecN<double2, 1> { using type = double2; };

// scatter: one thread per (distinct grid point, NB columns); alpha rows read as vectors.
template <typename T, int NB>
__global__ void __launch_bounds__(128)
    nl_scatter_kernel(T* __restrict__ out, long long ld, int ncol, int ncolp, NLView tab,
                      const T* __restrict__ alpha, typename ScalarOf<T>::type scale) {
    using S = typename ScalarOf<T>::type;
    constexpr int VW = 16 / sizeof(T);  // elements per 16-byte vector
    using VV = typename VecN<T, VW>::type;
    static_assert(NB % VW == 0, "column block must be a multiple of the vector width");
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
            const VV* al = reinterpret_cast<const VV*>(alpha + (long long)(poff + j) * ncolp + n0);
#pragma unroll
            for (int q = 0; q < NB / VW; ++q) {
                const VV v = __ldg(al + q);
                const T* ve = reinterpret_cast<const T*>(&v);
#pragma unroll
                for (int k = 0; k < VW; ++k) tmp[q * VW + k] = fmac(tmp[q * VW + k], c, ve[k]);
            }
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
