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
#include "kernels.h"
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
        if (j < np) {
            // Gamma dV as an FP32 (hi, lo) pair: a single rounded float would scale the projector's
            // channel by a fixed 1 + O(6e-8) and shift every Ritz value alike
            const double gd = tab.gamma[poff + j] * dV;
            const S hi = (S)gd;
            T v = vscale(hi, acc[m]);
            if (sizeof(S) == sizeof(float)) v = fmac(v, (S)(gd - (double)hi), acc[m]);
            alpha[(long long)(poff + j) * ncolp + n0 + n] = v;
        }
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

// ---------------------------------------------------------------------------------------------
// Register-tiled kernels for real (Gamma-point) data, T = float or double.
//
// gather2: CTA = (physical atom, 64 columns), 256 threads.  Point tiles of 64 sphere points are
// staged in shared memory: x as [point][column] with the 4-column groups XOR-swizzled by the
// point index (conflict-free stores from point-major loads and float4/double2 reads), chi as
// [point][two projector groups padded to 16 bytes].  Lane = (column group cg of 4 columns,
// projector group pg of NPG projectors), so every thread keeps 4 x NPG accumulators; the 8
// warps split the points of a tile and their partial sums are added in a fixed binary tree
// at the end (deterministic).
//
// scatter2: CTA = (image, 64 columns), 256 threads; images are launched one colour class at a
// time, and no two images of a class touch the same grid point, so every output element has
// one writer per launch and the summation order is fixed.  Warp w owns columns 8w..8w+7,
// lane owns 2 points of a 64-point tile; chi is staged [projector][point] and the atom's
// alpha block [projector][column] is read as broadcasts.
// ---------------------------------------------------------------------------------------------
constexpr int kNL2Cols = 64;  // columns per CTA of gather2 / scatter2
constexpr int kNL2Pts = kNLTilePts;  // points per staged tile

template <typename T>
__device__ __forceinline__ void load_vec4(const T* p, T (&v)[4]) {
    if constexpr (sizeof(T) == 4) {
        const float4 q = *reinterpret_cast<const float4*>(p);
        v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    } else {
        const double2 q0 = *reinterpret_cast<const double2*>(p);
        const double2 q1 = *reinterpret_cast<const double2*>(p + 2);
        v[0] = q0.x; v[1] = q0.y; v[2] = q1.x; v[3] = q1.y;
    }
}
template <typename T>
__device__ __forceinline__ void store_vec4(T* p, const T (&v)[4]) {
    if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
        *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
        *reinterpret_cast<double2*>(p + 2) = make_double2(v[2], v[3]);
    }
}

template <typename T, int NPG>
struct Gather2Geom {
    static constexpr int VW = 16 / sizeof(T);
    static constexpr int NPGP = (NPG + VW - 1) / VW * VW;  // projector group stride, 16-byte multiple
    static constexpr int CSP = 2 * NPGP;                   // chi row stride
    static constexpr size_t xs_elems = (size_t)kNL2Pts * kNL2Cols;
    static constexpr size_t cs_elems = (size_t)kNL2Pts * CSP;
    static constexpr size_t buf_elems = xs_elems + cs_elems;        // one tile buffer
    static constexpr size_t red_elems = (size_t)4 * 32 * 4 * NPG;  // 4 warps x 32 lanes x accumulators
    static constexpr size_t smem_bytes =
        sizeof(T) * ((2 * buf_elems) > red_elems ? (2 * buf_elems) : red_elems);
};

// Asynchronous 4- or 8-byte global -> shared copy; src_bytes = 0 fills the destination with
// zeros without reading the source.
template <int BYTES>
__device__ __forceinline__ void cp_async_small(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src), "n"(BYTES), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Position in an atom's tile sequence: image ii of the atom, first point g0 of the tile.
struct TileIt {
    int ii, g0;
};

// Tiles are double-buffered: the asynchronous copies of tile t+1 are issued before the FMAs of
// tile t, so the gathered loads of one tile overlap the arithmetic of the previous one.
template <typename T, int NPG>
__global__ void __launch_bounds__(256)
    nl_gather2_kernel(const T* __restrict__ x, long long ld, int ncol, int ncolp, NLView tab, T* __restrict__ alpha,
                      double dV) {
    using Geo = Gather2Geom<T, NPG>;
    constexpr int NB = kNL2Cols, G = kNL2Pts, NPGP = Geo::NPGP, CSP = Geo::CSP;
    extern __shared__ __align__(16) unsigned char smraw[];
    // two tile buffers, each [G][NB] x (4-column groups swizzled by g & 7) then [G][CSP] chi
    T* const buf0 = reinterpret_cast<T*>(smraw);
    const T* chi = reinterpret_cast<const T*>(tab.chi);
    const int a = blockIdx.x;
    const int n0 = blockIdx.y * NB;
    const int np = tab.atom_nproj[a];
    const int poff = tab.atom_poff[a];
    const int ii_end = tab.atom_img_ptr[a + 1];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int cg = lane & 15, pg = lane >> 4;
    T acc[4][NPG];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int m = 0; m < NPG; ++m) acc[k][m] = T(0);

    auto normalize = [&](TileIt t) {  // first non-empty tile at or after (ii, g0)
        while (t.ii < ii_end && t.g0 >= tab.img_ndc[tab.atom_img_list[t.ii]]) {
            ++t.ii;
            t.g0 = 0;
        }
        return t;
    };
    auto issue = [&](TileIt t, int bi) {  // asynchronous copies of tile t into buffer bi
        T* xs = buf0 + (size_t)bi * Geo::buf_elems;
        T* cs = xs + Geo::xs_elems;
        const int im = tab.atom_img_list[t.ii];
        const int ndc = tab.img_ndc[im];
        const int gl = min(G, ndc - t.g0);
        const int* gp = tab.gpos + tab.img_goff[im] + t.g0;
        const T* ch = chi + tab.img_chi_off[im] + t.g0;
#pragma unroll
        for (int pp = 0; pp < 2; ++pp) {
            const int g = lane + 32 * pp;
            const bool okg = g < gl;
            const long long base = okg ? (long long)gp[g] : 0;
#pragma unroll
            for (int qq = 0; qq < 2; ++qq) {
                const int q = w + 8 * qq;
                T* dst = xs + g * NB + 4 * (q ^ (g & 7));
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int col = n0 + 4 * q + k;
                    const bool ok = okg && col < ncol;
                    cp_async_small<sizeof(T)>(dst + k, x + (ok ? base + (long long)col * ld : 0),
                                              ok ? (int)sizeof(T) : 0);
                }
            }
        }
        for (int e = tid; e < G * CSP; e += 256) {
            const int g = e % G, sl = e / G;
            const int gq = sl / NPGP, m = sl % NPGP;
            const int j = gq * NPG + m;
            const bool ok = g < gl && m < NPG && j < np;
            cp_async_small<sizeof(T)>(cs + g * CSP + sl, ch + (ok ? (long long)j * ndc + g : 0),
                                      ok ? (int)sizeof(T) : 0);
        }
        cp_async_commit();
    };

    TileIt cur = normalize(TileIt{tab.atom_img_ptr[a], 0});
    int bi = 0;
    if (cur.ii < ii_end) issue(cur, 0);
    while (cur.ii < ii_end) {
        const int gl = min(G, tab.img_ndc[tab.atom_img_list[cur.ii]] - cur.g0);
        const TileIt nxt = normalize(TileIt{cur.ii, cur.g0 + G});
        if (nxt.ii < ii_end) {
            issue(nxt, bi ^ 1);  // that buffer was released by the barrier that ended the last tile
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const T* xs = buf0 + (size_t)bi * Geo::buf_elems;
        const T* cs = xs + Geo::xs_elems;
        for (int g = w; g < gl; g += 8) {
            T xv[4];
            load_vec4(xs + g * NB + 4 * (cg ^ (g & 7)), xv);
            const T* cp = cs + g * CSP + pg * NPGP;
            T cv[NPGP];
            if constexpr (sizeof(T) == 4) {
#pragma unroll
                for (int m = 0; m < NPGP; m += 4) {
                    const float4 q = *reinterpret_cast<const float4*>(cp + m);
                    cv[m] = q.x;
                    cv[m + 1] = q.y;
                    cv[m + 2] = q.z;
                    cv[m + 3] = q.w;
                }
            } else {
#pragma unroll
                for (int m = 0; m < NPGP; m += 2) {
                    const double2 q = *reinterpret_cast<const double2*>(cp + m);
                    cv[m] = q.x;
                    cv[m + 1] = q.y;
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int m = 0; m < NPG; ++m) acc[k][m] = fma(cv[m], xv[k], acc[k][m]);
        }
        __syncthreads();  // every warp is done with buffer bi before it is refilled
        cur = nxt;
        bi ^= 1;
    }
    // fixed-order tree over the 8 warps: 4+4, 2+2, 1+1
    T* red = reinterpret_cast<T*>(smraw);
#pragma unroll 1
    for (int h = 4; h >= 1; h >>= 1) {
        __syncthreads();
        if (w >= h && w < 2 * h) {
            T* r = red + ((size_t)(w - h) * 32 + lane) * (4 * NPG);
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int m = 0; m < NPG; ++m) r[k * NPG + m] = acc[k][m];
        }
        __syncthreads();
        if (w < h) {
            const T* r = red + ((size_t)w * 32 + lane) * (4 * NPG);
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int m = 0; m < NPG; ++m) acc[k][m] += r[k * NPG + m];
        }
    }
    if (w == 0) {
#pragma unroll
        for (int m = 0; m < NPG; ++m) {
            const int j = pg * NPG + m;
            if (j < np) {
                const double gd = tab.gamma[poff + j] * dV;  // applied as a (hi, lo) pair in FP32
                const T sc = (T)gd;
                const T sl = (T)(gd - (double)sc);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int col = n0 + 4 * cg + k;
                    if (col < ncolp) {
                        T v = sc * acc[k][m];
                        if (sizeof(T) == sizeof(float)) v = fma(sl, acc[k][m], v);
                        alpha[(long long)(poff + j) * ncolp + col] = v;
                    }
                }
            }
        }
    }
}

// COMPACT: instead of out[gpos] += scale * (chi alpha), store chi alpha into the compact
// per-point array out[col * ld + ent_pt[entry]] (every grid point has exactly one entry).
template <typename T, bool COMPACT = false>
__global__ void __launch_bounds__(256)
    nl_scatter2_kernel(T* __restrict__ out, long long ld, int ncol, int ncolp, NLView tab,
                       const int* __restrict__ imgs, const T* __restrict__ alpha, T scale,
                       const int* __restrict__ ent_pt = nullptr, const int2* __restrict__ tiles = nullptr) {
    constexpr int NB = kNL2Cols, G = kNL2Pts;
    extern __shared__ __align__(16) unsigned char smraw[];
    // tiles (optional): one CTA per (image, first point of a 64-point tile), so the read-modify-
    // write latencies of all tiles of a colour class overlap; otherwise one CTA per image.
    const int2 tl = tiles ? tiles[blockIdx.x] : make_int2(imgs[blockIdx.x], 0);
    const int im = tl.x;
    const int n0 = blockIdx.y * NB;
    const int a = tab.img_atom[im];
    const int np = tab.atom_nproj[a];
    const int poff = tab.atom_poff[a];
    const int ndc = tab.img_ndc[im];
    const int* gp = tab.gpos + tab.img_goff[im];
    const T* ch = reinterpret_cast<const T*>(tab.chi) + tab.img_chi_off[im];
    T* al = reinterpret_cast<T*>(smraw);  // [np][NB]
    T* cs = al + (size_t)np * NB;         // [np][G]
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int e = tid; e < np * NB; e += 256) {
        const int j = e / NB, c = e % NB;
        al[e] = (n0 + c < ncolp) ? alpha[(long long)(poff + j) * ncolp + n0 + c] : T(0);
    }
    const int gend = tiles ? min(ndc, tl.y + G) : ndc;
    for (int g0 = tl.y; g0 < gend; g0 += G) {
        __syncthreads();
        for (int e = tid; e < np * G; e += 256) {
            const int j = e / G, g = e % G;
            cs[e] = (g0 + g < ndc) ? ch[(long long)j * ndc + g0 + g] : T(0);
        }
        __syncthreads();
        T acc[2][8];
#pragma unroll
        for (int p = 0; p < 2; ++p)
#pragma unroll
            for (int k = 0; k < 8; ++k) acc[p][k] = T(0);
        for (int j = 0; j < np; ++j) {
            const T c0 = cs[j * G + lane], c1 = cs[j * G + lane + 32];
            T av[8];
            T t0[4], t1[4];
            load_vec4(al + j * NB + 8 * w, t0);
            load_vec4(al + j * NB + 8 * w + 4, t1);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                av[k] = t0[k];
                av[k + 4] = t1[k];
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                acc[0][k] = fma(c0, av[k], acc[0][k]);
                acc[1][k] = fma(c1, av[k], acc[1][k]);
            }
        }
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            const int g = g0 + lane + 32 * p;
            if (g < ndc) {
                if constexpr (COMPACT) {
                    T* o = out + ent_pt[tab.img_goff[im] + g];
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        const int col = n0 + 8 * w + k;
                        if (col < ncol) o[(long long)col * ld] = acc[p][k];
                    }
                } else {
                    T* o = out + gp[g];
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        const int col = n0 + 8 * w + k;
                        if (col < ncol) {
                            T* q = o + (long long)col * ld;
                            *q = fma(scale, acc[p][k], *q);
                        }
                    }
                }
            }
        }
    }
}

// expand on the compact numbering, point-major: W[col * ldw + pt] = sum_j chi_pt[j][pt] *
// alpha[(poff(atom(pt)) + j) * ncolp + col], summed over j in increasing order (the order the
// scatter kernels use).  CTA = 64 consecutive points x 64 columns, 256 threads: warp w owns
// columns 8w..8w+7, lane owns points lane and lane + 32, so every store instruction writes a
// contiguous run of W.
template <typename T>
__global__ void __launch_bounds__(256)
    nl_expand_pt_kernel(T* __restrict__ W, long long ldw, int ncol, int ncolp, int n_pts,
                        const T* __restrict__ chi_pt, const int2* __restrict__ pt_meta, const T* __restrict__ alpha) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int n0 = blockIdx.y * kNL2Cols + 8 * w;
    const int ptA = blockIdx.x * kNL2Pts + lane, ptB = ptA + 32;
    // pt_meta[pt] = (first projector row of the point's atom, projector count)
    const int2 mA = (ptA < n_pts) ? pt_meta[ptA] : make_int2(0, 0);
    const int2 mB = (ptB < n_pts) ? pt_meta[ptB] : make_int2(0, 0);
    const T* alA = alpha + (long long)mA.x * ncolp + n0;
    const T* alB = alpha + (long long)mB.x * ncolp + n0;
    const bool full = n0 + 8 <= ncolp;
    T accA[8], accB[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) accA[k] = accB[k] = T(0);
    auto row8 = [&](const T* al, int j, T (&v)[8]) {
        if (full) {
            T t0[4], t1[4];
            load_vec4(al + (long long)j * ncolp, t0);
            load_vec4(al + (long long)j * ncolp + 4, t1);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                v[k] = t0[k];
                v[k + 4] = t1[k];
            }
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = (n0 + k < ncolp) ? al[(long long)j * ncolp + k] : T(0);
        }
    };
    const int npm = max(mA.y, mB.y);
#pragma unroll 2
    for (int j = 0; j < npm; ++j) {
        if (j < mA.y) {
            const T c = chi_pt[(long long)j * n_pts + ptA];
            T v[8];
            row8(alA, j, v);
#pragma unroll
            for (int k = 0; k < 8; ++k) accA[k] = fma(c, v[k], accA[k]);
        }
        if (j < mB.y) {
            const T c = chi_pt[(long long)j * n_pts + ptB];
            T v[8];
            row8(alB, j, v);
#pragma unroll
            for (int k = 0; k < 8; ++k) accB[k] = fma(c, v[k], accB[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        if (n0 + k < ncol) {
            if (ptA < n_pts) W[(long long)(n0 + k) * ldw + ptA] = accA[k];
            if (ptB < n_pts) W[(long long)(n0 + k) * ldw + ptB] = accB[k];
        }
    }
}

// The same expansion, tiled.  CTA = one tile of kExpTilePts consecutive points (grid order) x
// CBN columns, 128 threads; thread = 4 consecutive points, so its stores of W are 16-byte
// vectors along the points and a warp writes 512 contiguous bytes per column.  The tile's chi
// values are staged in shared memory once, and the columns are swept in groups of VW (one
// 16-byte vector of alpha per (atom, projector)); the alpha vectors of the tile's atoms for the
// next group are fetched into registers while the current group is computed.  Neighbouring
// points mostly lie on one atom: a thread reads an alpha vector only where its points change
// atom, so shared-memory traffic is about a quarter of reading it per point.  NP (>= every
// atom's projector count) is a compile-time bound, so the projector loop unrolls and its
// shared-memory loads overlap.  Every (point, column) sums j = 0 .. NP-1 in order from zero
// (chi is zero past the atom's projector count), the order of the kernel above.
constexpr int kExpThreads = kExpTilePts / 4;
template <typename T, int NP>
__global__ void __launch_bounds__(kExpThreads)
    nl_expand_tile_kernel(T* __restrict__ W, long long ldw, int ncol, int ncolp, int n_pts,
                          const T* __restrict__ chi_pt, const unsigned char* __restrict__ pt_slot,
                          const int* __restrict__ tile_atoms, int amax, int max_np, const int* __restrict__ atom_poff,
                          const int* __restrict__ atom_nproj, const T* __restrict__ alpha) {
    constexpr int VW = 16 / (int)sizeof(T);  // columns per group (one 16-byte vector)
    constexpr int NG = 16;                   // groups per CTA
    constexpr int CBN = NG * VW;             // columns per CTA
    constexpr int PRE = 1024 / kExpThreads;  // alpha vectors a thread prefetches per group (amax * NP <= 1024)
    extern __shared__ __align__(16) unsigned char smx[];
    T* chi_s = reinterpret_cast<T*>(smx);                                              // [NP][kExpTilePts]
    float4* al_s = reinterpret_cast<float4*>(smx + (size_t)NP * kExpTilePts * sizeof(T));  // [2][amax * NP]
    const int t = blockIdx.x, tid = threadIdx.x;
    const long long p0 = (long long)t * kExpTilePts;
    const int* ta = tile_atoms + (long long)t * amax;
    const int nrow = amax * NP;  // alpha vectors of one group
    for (int e = tid; e < NP * kExpTilePts; e += kExpThreads) {
        const int j = e / kExpTilePts, q = e - j * kExpTilePts;
        const long long m = p0 + q;
        chi_s[e] = (m < n_pts && j < max_np) ? chi_pt[(long long)j * n_pts + m] : T(0);
    }
    // alpha vector r = slot * NP + j of column group g
    auto fetch = [&](int r, int g) {
        const int slot = r / NP, j = r - slot * NP;
        const int a = ta[slot];
        const int col = blockIdx.y * CBN + g * VW;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (a >= 0 && j < atom_nproj[a] && col < ncolp)
            v = *reinterpret_cast<const float4*>(alpha + (long long)(atom_poff[a] + j) * ncolp + col);
        return v;
    };
    float4 pre[PRE];
#pragma unroll
    for (int i = 0; i < PRE; ++i)
        if (tid + kExpThreads * i < nrow) pre[i] = fetch(tid + kExpThreads * i, 0);
    const long long m0 = p0 + 4 * tid;
    int sl[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) sl[k] = (m0 + k < n_pts) ? (int)pt_slot[m0 + k] * NP : 0;
    for (int g = 0; g < NG; ++g) {
        const int col0 = blockIdx.y * CBN + g * VW;
        if (col0 >= ncol) break;
        float4* al = al_s + (size_t)(g & 1) * nrow;
#pragma unroll
        for (int i = 0; i < PRE; ++i)
            if (tid + kExpThreads * i < nrow) al[tid + kExpThreads * i] = pre[i];
        __syncthreads();  // the group's alpha vectors (and, at g = 0, the chi tile) are staged
        if (g + 1 < NG) {
#pragma unroll
            for (int i = 0; i < PRE; ++i)
                if (tid + kExpThreads * i < nrow) pre[i] = fetch(tid + kExpThreads * i, g + 1);
        }
        T acc[4][VW];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int c = 0; c < VW; ++c) acc[k][c] = T(0);
#pragma unroll
        for (int j = 0; j < NP; ++j) {
            T cj[4];
            const float4* cs = reinterpret_cast<const float4*>(chi_s + (size_t)j * kExpTilePts + 4 * tid);
#pragma unroll
            for (int h = 0; h < (int)(4 * sizeof(T) / 16); ++h) reinterpret_cast<float4*>(cj)[h] = cs[h];
            float4 raw = al[sl[0] + j];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (k > 0 && sl[k] != sl[k - 1]) raw = al[sl[k] + j];
                const T* v = reinterpret_cast<const T*>(&raw);
#pragma unroll
                for (int c = 0; c < VW; ++c) acc[k][c] = fma(cj[k], v[c], acc[k][c]);
            }
        }
        if (m0 + 3 < n_pts) {
#pragma unroll
            for (int c = 0; c < VW; ++c)
                if (col0 + c < ncol) {
                    T o[4] = {acc[0][c], acc[1][c], acc[2][c], acc[3][c]};
                    T* dst = W + (long long)(col0 + c) * ldw + m0;
                    if constexpr (sizeof(T) == 4) {
                        *reinterpret_cast<float4*>(dst) = *reinterpret_cast<const float4*>(o);
                    } else {
                        reinterpret_cast<double2*>(dst)[0] = make_double2(o[0], o[1]);
                        reinterpret_cast<double2*>(dst)[1] = make_double2(o[2], o[3]);
                    }
                }
        } else {
#pragma unroll
            for (int c = 0; c < VW; ++c)
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (col0 + c < ncol && m0 + k < n_pts) W[(long long)(col0 + c) * ldw + m0 + k] = acc[k][c];
        }
    }
}

// The same expansion with the projector values in registers and alpha in shared memory.
// CTA = one tile of kExpTilePts consecutive points (grid order) x kExpRegCols columns; thread =
// PTS consecutive points (one 16-byte vector of W per column: 4 floats or 2 doubles), whose chi
// values it loads once into registers.  The alpha rows of the tile's atoms for the CTA's columns
// are staged in shared memory with one barrier, [slot][projector][column]; the thread then
// sweeps the columns in groups of VW (one 16-byte alpha vector per projector, re-read only where
// its points change atom, so one shared-memory load serves up to PTS x VW outputs) and writes W
// as 16-byte vectors (a warp writes 512 contiguous bytes per column).  Every (point, column)
// sums j = 0 .. NP-1 in order from zero with fma (chi and alpha are zero past the atom's
// projector count), the order of the kernels above: bitwise their results.  FP32 column pairs
// use packed fma.rn.f32x2, element for element the same rounding.
constexpr int kExpRegCols = 32;
template <typename T>
constexpr int exp_reg_threads() {
    return kExpTilePts / (16 / (int)sizeof(T));
}
template <typename T, int NP>
__global__ void __launch_bounds__(exp_reg_threads<T>())
    nl_expand_reg_kernel(T* __restrict__ W, long long ldw, int ncol, int ncolp, int n_pts, int max_np,
                         const T* __restrict__ chi_pt, const unsigned char* __restrict__ pt_slot,
                         const int* __restrict__ tile_atoms, int amax, const int* __restrict__ atom_poff,
                         const int* __restrict__ atom_nproj, const T* __restrict__ alpha) {
    constexpr int PTS = 16 / (int)sizeof(T);   // points per thread
    constexpr int VW = 16 / (int)sizeof(T);    // columns per alpha vector
    constexpr int NV = kExpRegCols / VW;       // alpha vectors per (slot, projector) row
    constexpr int NT = exp_reg_threads<T>();
    constexpr bool kF32 = std::is_same<T, float>::value;
    using V16 = typename std::conditional<kF32, float4, double2>::type;
    extern __shared__ __align__(16) unsigned char smx[];
    // [amax][NP][NV] with the slot stride padded by one vector: the points of a warp span several
    // atoms (runs of ~8 points alternate between atoms along a row), and unpadded slot rows would
    // all start on the same banks
    constexpr int SS = NP * NV + 1;
    V16* al_s = reinterpret_cast<V16*>(smx);
    const int t = blockIdx.x, tid = threadIdx.x;
    const int c0 = blockIdx.y * kExpRegCols;
    const int* ta = tile_atoms + (long long)t * amax;
    for (int e = tid; e < amax * NP * NV; e += NT) {
        const int r = e / NV, v = e - r * NV;
        const int slot = r / NP, j = r - slot * NP;
        const int a = ta[slot];
        const int col = c0 + v * VW;
        V16 val;
        T* vp = reinterpret_cast<T*>(&val);
#pragma unroll
        for (int c = 0; c < VW; ++c) vp[c] = T(0);
        if (a >= 0 && j < atom_nproj[a] && col < ncolp)
            val = *reinterpret_cast<const V16*>(alpha + (long long)(atom_poff[a] + j) * ncolp + col);
        al_s[slot * SS + j * NV + v] = val;
    }
    const long long m0 = (long long)t * kExpTilePts + PTS * tid;
    const int npt = (int)max(0LL, min((long long)PTS, (long long)n_pts - m0));
    T cj[NP][PTS];
    const bool vec = npt == PTS && (n_pts % PTS) == 0;  // chi rows 16-byte aligned at m0
#pragma unroll
    for (int j = 0; j < NP; ++j) {
        const T* src = chi_pt + (long long)j * n_pts + m0;
        if (j < max_np && vec) {
            const V16 q = *reinterpret_cast<const V16*>(src);
            const T* qp = reinterpret_cast<const T*>(&q);
#pragma unroll
            for (int k = 0; k < PTS; ++k) cj[j][k] = qp[k];
        } else {
#pragma unroll
            for (int k = 0; k < PTS; ++k) cj[j][k] = (j < max_np && k < npt) ? src[k] : T(0);
        }
    }
    int so[PTS];  // each point's slot row in al_s (past the last point: the previous one's)
#pragma unroll
    for (int k = 0; k < PTS; ++k) so[k] = (k < npt) ? (int)pt_slot[m0 + k] * SS : (k > 0 ? so[k - 1] : 0);
    __syncthreads();  // alpha staged
    if (npt == 0) return;
#pragma unroll 1
    for (int g = 0; g < NV; ++g) {
        const int col = c0 + g * VW;
        if (col >= ncol) break;
        T acc[PTS][VW];
#pragma unroll
        for (int k = 0; k < PTS; ++k)
#pragma unroll
            for (int c = 0; c < VW; ++c) acc[k][c] = T(0);
#pragma unroll
        for (int j = 0; j < NP; ++j) {
            V16 av = al_s[so[0] + j * NV + g];
#pragma unroll
            for (int k = 0; k < PTS; ++k) {
                if (k > 0 && so[k] != so[k - 1]) av = al_s[so[k] + j * NV + g];
                const T* v = reinterpret_cast<const T*>(&av);
                if constexpr (kF32) {
                    const float2 x = make_float2(cj[j][k], cj[j][k]);
#pragma unroll
                    for (int c = 0; c < VW; c += 2) {
                        const float2 r = __ffma2_rn(x, make_float2(v[c], v[c + 1]), make_float2(acc[k][c], acc[k][c + 1]));
                        acc[k][c] = r.x;
                        acc[k][c + 1] = r.y;
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < VW; ++c) acc[k][c] = fma(cj[j][k], v[c], acc[k][c]);
                }
            }
        }
#pragma unroll
        for (int c = 0; c < VW; ++c) {
            if (col + c >= ncol) break;
            T* dst = W + (long long)(col + c) * ldw + m0;
            if (npt == PTS) {
                V16 o;
                T* op = reinterpret_cast<T*>(&o);
#pragma unroll
                for (int k = 0; k < PTS; ++k) op[k] = acc[k][c];
                *reinterpret_cast<V16*>(dst) = o;
            } else {
#pragma unroll
                for (int k = 0; k < PTS; ++k)
                    if (k < npt) dst[k] = acc[k][c];
            }
        }
    }
}

// Nonlocal force reduction for one direction (src/physics/Forces.cpp:772-777, :682-684):
//   force[a * 3 + dim] = -spn * sum_n occ[n] sum_{j < np(a)} Gamma[poff+j] Re(conj(alpha) beta)
// and, for dim == 0, the atom's energy share  ea[a] = efac * sum_n occ[n] sum_j Gamma |alpha|^2.
// alpha, beta: projections without Gamma, [total_proj][ncolp].  CTA = atom; fixed-order sums.
__device__ __forceinline__ double re_conj_mul(double a, double b) { return a * b; }
__device__ __forceinline__ double re_conj_mul(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }

template <typename T>
__global__ void __launch_bounds__(256)
    nl_force_reduce_kernel(const T* __restrict__ alpha, const T* __restrict__ beta, int ncolp, int ncol,
                           const double* __restrict__ occ, const int* __restrict__ atom_nproj,
                           const int* __restrict__ atom_poff, const double* __restrict__ gamma, double spn,
                           double efac, int dim, double* __restrict__ force, double* __restrict__ ea) {
    __shared__ double rf[256], re[256];
    const int a = blockIdx.x;
    const int np = atom_nproj[a], poff = atom_poff[a];
    double sf = 0.0, se = 0.0;
    for (int e = threadIdx.x; e < np * ncol; e += blockDim.x) {
        const int j = e / ncol, n = e % ncol;
        const long long o = (long long)(poff + j) * ncolp + n;
        const double w = occ[n] * gamma[poff + j];
        sf += w * re_conj_mul(alpha[o], beta[o]);
        if (dim == 0) se += w * re_conj_mul(alpha[o], alpha[o]);
    }
    rf[threadIdx.x] = sf;
    re[threadIdx.x] = se;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            rf[threadIdx.x] += rf[threadIdx.x + h];
            re[threadIdx.x] += re[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        force[a * 3 + dim] = -spn * rf[0];
        if (dim == 0) ea[a] = efac * re[0];
    }
}

}  // namespace lynxb
