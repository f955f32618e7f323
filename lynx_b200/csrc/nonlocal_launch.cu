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
}  // namespace

template <typename T>
int launch_nl_gather(const NLDev& nl, const T* x, long long ld, int ncol, T* alpha, int ncolp, double dV,
                     cudaStream_t st) {
    using S = typename ScalarOf<T>::type;
    constexpr int NB = 32;  // columns per CTA; 8 projector groups of 256 threads
    static_assert(kNLColBlock % 16 == 0 && NB % kNLColBlock == 0 || kNLColBlock % NB == 0, "column blocks");
    if (nl.n_atom == 0 || ncol <= 0) return LYNX_OK;
    const int pj = (nl.max_np + 7) / 8;
    if (pj > 4) {
        set_error("%d projectors per atom exceed the gather kernel's limit of 32", nl.max_np);
        return LYNX_ERR_UNSUPPORTED;
    }
    const size_t smem = sizeof(T) * kGatherTile * (NB + 1) + sizeof(S) * nl.max_np * kGatherTile;
    dim3 grid(nl.n_atom, (ncol + NB - 1) / NB);
    auto go = [&](auto kern) {
        if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
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

template int launch_nl_gather<double>(const NLDev&, const double*, long long, int, double*, int, double, cudaStream_t);
template int launch_nl_gather<float>(const NLDev&, const float*, long long, int, float*, int, double, cudaStream_t);
template int launch_nl_gather<double2>(const NLDev&, const double2*, long long, int, double2*, int, double, cudaStream_t);
template int launch_nl_gather<float2>(const NLDev&, const float2*, long long, int, float2*, int, double, cudaStream_t);
template int launch_nl_scatter<double, double>(const NLDev&, double*, long long, int, const double*, int, double, cudaStream_t);
template int launch_nl_scatter<float, float>(const NLDev&, float*, long long, int, const float*, int, float, cudaStream_t);
template int launch_nl_scatter<double2, double>(const NLDev&, double2*, long long, int, const double2*, int, double, cudaStream_t);
template int launch_nl_scatter<float2, float>(const NLDev&, float2*, long long, int, const float2*, int, float, cudaStream_t);

}  // namespace lynxb
