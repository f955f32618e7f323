// Launchers for the deterministic nonlocal gather / scatter kernels.
#include <type_traits>
#include "kernels.h"
#include "lynx_common.cuh"
#include "nonlocal.cuh"

namespace lynxb {

namespace {
template <typename T>
NLView make_view(const NLDev& nl) {
    NLView v;
    v.n_atom = nl.n_atom;
    v.n_img = nl.n_img;
    v.n_pts = nl.n_pts;
    v.atom_img_ptr = nl.atom_img_ptr;
    v.atom_img_list = nl.atom_img_list;
    v.atom_nproj = nl.atom_nproj;
    v.atom_poff = nl.atom_poff;
    v.gamma = nl.gamma;
    v.img_atom = nl.img_atom;
    v.img_ndc = nl.img_ndc;
    v.img_goff = nl.img_goff;
    v.img_chi_off = nl.img_chi_off;
    v.img_phase = nl.img_phase;
    v.gpos = nl.gpos;
    v.chi = std::is_same<typename ScalarOf<T>::type, float>::value ? (const void*)nl.chi32 : (const void*)nl.chi64;
    v.pt_grid = nl.pt_grid;
    v.pt_ptr = nl.pt_ptr;
    v.ent_img = nl.ent_img;
    v.ent_loc = nl.ent_loc;
    return v;
}
template <typename T>
constexpr bool kReal = std::is_same<T, float>::value || std::is_same<T, double>::value;

int launch_status(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s launch failed: %s", what, cudaGetErrorString(e));
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

template <typename T, int NPG>
int gather2(const NLDev& nl, const T* x, long long ld, int ncol, T* alpha, int ncolp, double dV, cudaStream_t st) {
    const size_t smem = Gather2Geom<T, NPG>::smem_bytes;
    auto kern = nl_gather2_kernel<T, NPG>;
    LYNX_CUDA_TRY(smem_cap(kern, smem));
    dim3 grid(nl.n_atom, (ncol + kNL2Cols - 1) / kNL2Cols);
    kern<<<grid, 256, smem, st>>>(x, ld, ncol, ncolp, make_view<T>(nl), alpha, dV);
    count_launch();
    return launch_status("nonlocal gather");
}

// Register-tiled gather for real data: projector groups of NPG >= ceil(max_np / 2).
template <typename T>
int gather2_dispatch(const NLDev& nl, const T* x, long long ld, int ncol, T* alpha, int ncolp, double dV,
                     cudaStream_t st) {
    const int h = (nl.max_np + 1) / 2;
    if (h <= 1) return gather2<T, 1>(nl, x, ld, ncol, alpha, ncolp, dV, st);
    if (h <= 2) return gather2<T, 2>(nl, x, ld, ncol, alpha, ncolp, dV, st);
    if (h <= 4) return gather2<T, 4>(nl, x, ld, ncol, alpha, ncolp, dV, st);
    if (h <= 5) return gather2<T, 5>(nl, x, ld, ncol, alpha, ncolp, dV, st);
    if (h <= 8) return gather2<T, 8>(nl, x, ld, ncol, alpha, ncolp, dV, st);
    if (h <= 9) return gather2<T, 9>(nl, x, ld, ncol, alpha, ncolp, dV, st);
    if (h <= 12) return gather2<T, 12>(nl, x, ld, ncol, alpha, ncolp, dV, st);
    return gather2<T, 16>(nl, x, ld, ncol, alpha, ncolp, dV, st);
}
}  // namespace

template <typename T>
int launch_nl_gather(const NLDev& nl, const T* x, long long ld, int ncol, T* alpha, int ncolp, double dV,
                     cudaStream_t st) {
    using S = typename ScalarOf<T>::type;
    constexpr int NB = 32;  // columns per CTA; 8 projector groups of 256 threads
    static_assert(kNLColBlock % 16 == 0 && NB % kNLColBlock == 0 || kNLColBlock % NB == 0, "column blocks");
    if (nl.n_atom == 0 || ncol <= 0) return LYNX_OK;
    if constexpr (kReal<T>) {
        if (nl.max_np <= 32) return gather2_dispatch<T>(nl, x, ld, ncol, alpha, ncolp, dV, st);
    }
    const int pj = (nl.max_np + 7) / 8;
    if (pj > 4) {
        set_error("%d projectors per atom exceed the gather kernel's limit of 32", nl.max_np);
        return LYNX_ERR_UNSUPPORTED;
    }
    const size_t smem = sizeof(T) * kGatherTile * (NB + 1) + sizeof(S) * nl.max_np * kGatherTile;
    dim3 grid(nl.n_atom, (ncol + NB - 1) / NB);
    auto go = [&](auto kern) {
        smem_cap(kern, smem);
        kern<<<grid, 256, smem, st>>>(x, ld, ncol, ncolp, make_view<T>(nl), alpha, dV);
    };
    if (pj <= 1) go(nl_gather_kernel<T, NB, 1>);
    else if (pj == 2) go(nl_gather_kernel<T, NB, 2>);
    else if (pj == 3) go(nl_gather_kernel<T, NB, 3>);
    else go(nl_gather_kernel<T, NB, 4>);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("nonlocal gather launch failed: %s", cudaGetErrorString(e));
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

template <typename T, typename S>
int launch_nl_scatter(const NLDev& nl, T* out, long long ld, int ncol, const T* alpha, int ncolp, S scale,
                      cudaStream_t st) {
    constexpr int NB = 16;
    if (nl.n_pts == 0 || ncol <= 0) return LYNX_OK;
    if constexpr (kReal<T>) {
        if (nl.n_colors > 0 && nl.max_np <= 32) {
            const size_t smem = sizeof(T) * 2 * (size_t)nl.max_np * kNL2Cols;
            for (int k = 0; k < nl.n_colors; ++k) {
                const int cnt = nl.color_toff[k + 1] - nl.color_toff[k];
                if (cnt == 0) continue;
                dim3 grid(cnt, (ncol + kNL2Cols - 1) / kNL2Cols);
                nl_scatter2_kernel<T><<<grid, 256, smem, st>>>(out, ld, ncol, ncolp, make_view<T>(nl), nullptr, alpha,
                                                               (T)scale, nullptr, nl.color_tiles + nl.color_toff[k]);
                count_launch();
                LYNX_TRY(launch_status("nonlocal scatter"));
            }
            return LYNX_OK;
        }
    }
    dim3 grid((nl.n_pts + 127) / 128, (ncol + NB - 1) / NB);
    nl_scatter_kernel<T, NB><<<grid, 128, 0, st>>>(out, ld, ncol, ncolp, make_view<T>(nl), alpha, scale);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("nonlocal scatter launch failed: %s", cudaGetErrorString(e));
        return LYNX_ERR_CUDA;
    }
    return LYNX_OK;
}

template <typename T>
int launch_nl_expand(const NLDev& nl, T* W, long long ldw, int ncol, const T* alpha, int ncolp, cudaStream_t st) {
    if constexpr (kReal<T>) {
        if (!nl.compact || nl.n_colors != 1 || nl.max_np > 32) {
            set_error("compact nonlocal expansion needs disjoint projector spheres");
            return LYNX_ERR_UNSUPPORTED;
        }
        if (nl.n_pts == 0 || ncol <= 0) return LYNX_OK;
        const T* chi_pt;
        if constexpr (std::is_same<T, float>::value) chi_pt = nl.chi_pt32;
        else chi_pt = nl.chi_pt64;
        constexpr int CBN = 16 * (16 / (int)sizeof(T));  // columns per CTA of the tile kernel
        // projector-count bound of the compiled instantiations
        const int NP = nl.max_np <= 4 ? 4 : nl.max_np <= 9 ? 9 : nl.max_np <= 18 ? 18 : 32;
        const size_t nrow = (size_t)nl.exp_amax * NP;
        const size_t smem = (size_t)NP * kExpTilePts * sizeof(T) + 2 * nrow * 16;
        const size_t smem_reg = (size_t)nl.exp_amax * (NP * kExpRegCols * sizeof(T) + 16);
        if (NP <= 18 && nl.exp_tile_atoms && smem_reg <= 96 * 1024 && (ldw % 4) == 0) {
            // projector values in registers (up to 18 per point), alpha staged in shared memory
            dim3 grid((nl.n_pts + kExpTilePts - 1) / kExpTilePts, (ncol + kExpRegCols - 1) / kExpRegCols);
            auto go = [&](auto kern) -> int {
                LYNX_CUDA_TRY(smem_cap(kern, smem_reg));
                kern<<<grid, exp_reg_threads<T>(), smem_reg, st>>>(W, ldw, ncol, ncolp, nl.n_pts, nl.max_np, chi_pt,
                                                             nl.pt_slot, nl.exp_tile_atoms, nl.exp_amax, nl.atom_poff,
                                                             nl.atom_nproj, alpha);
                return LYNX_OK;
            };
            if (NP == 4) LYNX_TRY(go(nl_expand_reg_kernel<T, 4>));
            else if (NP == 9) LYNX_TRY(go(nl_expand_reg_kernel<T, 9>));
            else LYNX_TRY(go(nl_expand_reg_kernel<T, 18>));
        } else if (nl.exp_tile_atoms && nrow <= 1024 && smem <= 200 * 1024 && (ldw % 4) == 0) {
            dim3 grid((nl.n_pts + kExpTilePts - 1) / kExpTilePts, (ncol + CBN - 1) / CBN);
            auto go = [&](auto kern) -> int {
                LYNX_CUDA_TRY(smem_cap(kern, smem));
                kern<<<grid, kExpThreads, smem, st>>>(W, ldw, ncol, ncolp, nl.n_pts, chi_pt, nl.pt_slot,
                                                      nl.exp_tile_atoms, nl.exp_amax, nl.max_np, nl.atom_poff,
                                                      nl.atom_nproj, alpha);
                return LYNX_OK;
            };
            if (NP == 4) LYNX_TRY(go(nl_expand_tile_kernel<T, 4>));
            else if (NP == 9) LYNX_TRY(go(nl_expand_tile_kernel<T, 9>));
            else if (NP == 18) LYNX_TRY(go(nl_expand_tile_kernel<T, 18>));
            else LYNX_TRY(go(nl_expand_tile_kernel<T, 32>));
        } else {
            dim3 grid((nl.n_pts + kNL2Pts - 1) / kNL2Pts, (ncol + kNL2Cols - 1) / kNL2Cols);
            nl_expand_pt_kernel<T><<<grid, 256, 0, st>>>(W, ldw, ncol, ncolp, nl.n_pts, chi_pt, nl.pt_meta, alpha);
        }
        count_launch();
        return launch_status("nonlocal expansion");
    } else {
        set_error("compact nonlocal expansion is for real data");
        return LYNX_ERR_UNSUPPORTED;
    }
}

template <typename T>
int launch_nl_force_reduce(const NLDev& nl, const T* alpha, const T* beta, int ncolp, int ncol, const double* occ,
                           double spn, double efac, int dim, double* force, double* ea, cudaStream_t st) {
    if (nl.n_atom == 0 || ncol <= 0) return LYNX_OK;
    nl_force_reduce_kernel<T><<<nl.n_atom, 256, 0, st>>>(alpha, beta, ncolp, ncol, occ, nl.atom_nproj, nl.atom_poff,
                                                         nl.gamma, spn, efac, dim, force, ea);
    count_launch();
    return launch_status("nonlocal force reduction");
}
template int launch_nl_force_reduce<double>(const NLDev&, const double*, const double*, int, int, const double*, double,
                                            double, int, double*, double*, cudaStream_t);
template int launch_nl_force_reduce<double2>(const NLDev&, const double2*, const double2*, int, int, const double*,
                                             double, double, int, double*, double*, cudaStream_t);

template int launch_nl_expand<double>(const NLDev&, double*, long long, int, const double*, int, cudaStream_t);
template int launch_nl_expand<float>(const NLDev&, float*, long long, int, const float*, int, cudaStream_t);
template int launch_nl_gather<double>(const NLDev&, const double*, long long, int, double*, int, double, cudaStream_t);
template int launch_nl_gather<float>(const NLDev&, const float*, long long, int, float*, int, double, cudaStream_t);
template int launch_nl_gather<double2>(const NLDev&, const double2*, long long, int, double2*, int, double, cudaStream_t);
template int launch_nl_gather<float2>(const NLDev&, const float2*, long long, int, float2*, int, double, cudaStream_t);
template int launch_nl_scatter<double, double>(const NLDev&, double*, long long, int, const double*, int, double, cudaStream_t);
template int launch_nl_scatter<float, float>(const NLDev&, float*, long long, int, const float*, int, float, cudaStream_t);
template int launch_nl_scatter<double2, double>(const NLDev&, double2*, long long, int, const double2*, int, double, cudaStream_t);
template int launch_nl_scatter<float2, float>(const NLDev&, float2*, long long, int, const float2*, int, float, cudaStream_t);

}  // namespace lynxb
