// Test-oracle harness around the reference LYNX CPU hot path (and the forces, stress and density
// that consume its orbitals).
//
// This file is TEST INFRASTRUCTURE.  It is compiled together with the
// reference's own, unmodified sources (src/solvers/EigenSolver.cpp,
// src/operators/Hamiltonian.cpp, src/operators/NonlocalProjector.cpp,
// src/parallel/HaloExchange.cpp, src/operators/FDStencil.cpp, src/atoms/*,
// src/core/{Lattice,FDGrid,Domain,KPoints,NumericalMethods}.cpp,
// src/electronic/Occupation.cpp) by oracle/Makefile into oracle/_ref/libref_lynx.so.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it,
// and only as the checker / the timed CPU reference.  Nothing in lynx_b200/
// links or calls it.
//
// The reference classes keep their state private and are normally wired up by
// the LynxContext singleton (src/core/LynxContext.cpp), which needs a full JSON
// system description, libxc and MPI.  The harness instead builds the same
// objects directly (Lattice -> FDGrid -> Domain -> FDStencil -> HaloExchange ->
// Crystal/NonlocalProjector -> Hamiltonian -> EigenSolver) and sets the three
// EigenSolver back-pointers that EigenSolver::setup (src/solvers/EigenSolver.cpp:160)
// would set, which is why private members are made reachable below.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <vector>
#include <mpi.h>
#include <omp.h>

#define private public
#define protected public
#include "atoms/Crystal.hpp"
#include "core/Domain.hpp"
#include "core/LynxContext.hpp"
#include "electronic/ElectronDensity.hpp"
#include "electronic/Wavefunction.hpp"
#include "operators/Gradient.hpp"
#include "operators/Laplacian.hpp"
#include "solvers/PoissonSolver.hpp"
#include "parallel/Parallelization.hpp"
#include "physics/Forces.hpp"
#include "physics/Stress.hpp"
#include "core/FDGrid.hpp"
#include "core/KPoints.hpp"
#include "core/Lattice.hpp"
#include "electronic/Occupation.hpp"
#include "operators/FDStencil.hpp"
#include "operators/Hamiltonian.hpp"
#include "operators/NonlocalProjector.hpp"
#include "parallel/HaloExchange.hpp"
#include "solvers/EigenSolver.hpp"
#include "solvers/Lanczos.hpp"
#include "xc/ExactExchange.hpp"
#undef private
#undef protected

using lynx::Complex;
using lynx::Vec3;

namespace {

struct RefState {
    lynx::Lattice lattice;
    lynx::FDGrid grid;
    lynx::Domain domain;
    lynx::FDStencil stencil;
    lynx::HaloExchange halo;
    std::unique_ptr<lynx::Crystal> crystal;
    std::vector<lynx::AtomNlocInfluence> nloc;
    lynx::NonlocalProjector vnl;
    bool has_vnl = false;
    lynx::Hamiltonian H;
    lynx::EigenSolver es;
    Vec3 kpt{0, 0, 0};
};

RefState* g = nullptr;
std::string g_err;

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void ref_free() {
    delete g;
    g = nullptr;
}

// latvec: 3x3 row-major, rows = lattice vectors (Bohr).  orth != 0 selects
// CellType::Orthogonal.  pos: natom x 3 atom positions in the coordinates the
// reference's Crystal expects (Cartesian for orthogonal cells, non-Cartesian
// "scaled fractional" for non-orthogonal ones, src/atoms/Crystal.cpp:25-41).
// psp8_path may be NULL or empty: then no nonlocal projector is set up.
// bc: 3 ints, 0 = BCType::Periodic, 1 = BCType::Dirichlet (src/core/types.hpp:14), or NULL
// for a periodic cell.
int ref_setup_bc(const double* latvec, int orth, int Nx, int Ny, int Nz, int fd_order,
                 int natom, const double* pos, const char* psp8_path, const int* bc) {
    return guarded([&] {
        ref_free();
        g = new RefState();
        lynx::Mat3 L;
        for (int i = 0; i < 9; ++i) L.data[i] = latvec[i];
        g->lattice = lynx::Lattice(L, orth ? lynx::CellType::Orthogonal : lynx::CellType::NonOrthogonal);
        auto bct = [&](int d) { return (bc && bc[d]) ? lynx::BCType::Dirichlet : lynx::BCType::Periodic; };
        g->grid = lynx::FDGrid(Nx, Ny, Nz, g->lattice, bct(0), bct(1), bct(2));
        lynx::DomainVertices v;
        v.xs = 0; v.xe = Nx - 1; v.ys = 0; v.ye = Ny - 1; v.zs = 0; v.ze = Nz - 1;
        g->domain = lynx::Domain(g->grid, v);
        g->stencil = lynx::FDStencil(fd_order, g->grid, g->lattice);
        g->halo = lynx::HaloExchange(g->domain, fd_order / 2);
        g->has_vnl = false;
        if (psp8_path && psp8_path[0] && natom > 0) {
            std::vector<lynx::AtomType> types;
            types.emplace_back("Si", 28.0855, 4.0, natom);
            types[0].psd().load_psp8(psp8_path);
            std::vector<Vec3> P;
            std::vector<int> ti;
            for (int a = 0; a < natom; ++a) {
                P.push_back(Vec3(pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]));
                ti.push_back(0);
            }
            g->crystal.reset(new lynx::Crystal(std::move(types), std::move(P), std::move(ti), g->lattice));
            g->crystal->compute_nloc_influence(g->domain, g->nloc);
            g->vnl.setup(*g->crystal, g->nloc, g->domain, g->grid);
            g->has_vnl = true;
        }
        g->H.setup(g->stencil, g->domain, g->grid, g->halo, g->has_vnl ? &g->vnl : nullptr);
        if (g->has_vnl) g->H.set_vnl_kpt(&g->vnl);
        // What EigenSolver::setup (src/solvers/EigenSolver.cpp:160-176) sets, minus MPI.
        g->es.H_ = &g->H;
        g->es.halo_ = &g->halo;
        g->es.domain_ = &g->domain;
        g->es.npband_ = 1;
    });
}

int ref_setup(const double* latvec, int orth, int Nx, int Ny, int Nz, int fd_order, int natom, const double* pos,
              const char* psp8_path) {
    return ref_setup_bc(latvec, orth, Nx, Ny, Nz, fd_order, natom, pos, psp8_path, nullptr);
}

int ref_nd() { return g ? g->domain.Nd_d() : 0; }
double ref_dV() { return g ? g->grid.dV() : 0.0; }

// Stencil coefficients (FDn+1 each) and the max eigenvalue of -0.5*Lap.
int ref_stencil(double* d2x, double* d2y, double* d2z, double* d1x, double* d1y, double* d1z,
                double* d2xy, double* d2xz, double* d2yz, double* maxeig, double* w1, double* w2) {
    if (!g) return -1;
    int n = g->stencil.FDn() + 1;
    auto cp = [n](double* dst, const double* src) {
        if (dst) std::memcpy(dst, src, n * sizeof(double));
    };
    cp(d2x, g->stencil.D2_coeff_x());
    cp(d2y, g->stencil.D2_coeff_y());
    cp(d2z, g->stencil.D2_coeff_z());
    cp(d1x, g->stencil.D1_coeff_x());
    cp(d1y, g->stencil.D1_coeff_y());
    cp(d1z, g->stencil.D1_coeff_z());
    cp(d2xy, g->stencil.D2_coeff_xy());
    cp(d2xz, g->stencil.D2_coeff_xz());
    cp(d2yz, g->stencil.D2_coeff_yz());
    cp(w1, g->stencil.weights_D1());
    cp(w2, g->stencil.weights_D2());
    if (maxeig) *maxeig = g->stencil.max_eigval_half_lap();
    return 0;
}

// Lattice-derived matrices: lapc_T (3x3), lat_uvec (3x3), jacobian.
int ref_lattice(double* lapcT, double* uvec, double* jac, double* lengths) {
    if (!g) return -1;
    if (lapcT) std::memcpy(lapcT, g->lattice.lapc_T().data, 9 * sizeof(double));
    if (uvec) std::memcpy(uvec, g->lattice.lat_uvec().data, 9 * sizeof(double));
    if (jac) *jac = g->lattice.jacobian();
    if (lengths) {
        Vec3 l = g->lattice.lengths();
        lengths[0] = l.x; lengths[1] = l.y; lengths[2] = l.z;
    }
    return 0;
}

// Nonlocal influence sizes: number of atom images with a non-empty sphere,
// total grid points over all images, projectors per atom, physical atoms.
int ref_nl_counts(int* n_img, int* total_ndc, int* nproj, int* n_atom) {
    if (!g) return -1;
    *n_img = 0; *total_ndc = 0; *nproj = 0; *n_atom = 0;
    if (!g->has_vnl) return 0;
    const auto& inf = g->nloc[0];
    *n_img = inf.n_atom;
    for (int i = 0; i < inf.n_atom; ++i) *total_ndc += inf.ndc[i];
    *nproj = g->crystal->types()[0].psd().nproj_per_atom();
    *n_atom = g->crystal->n_atom_total();
    return 0;
}

// Flattened projector tables in the order the reference iterates them
// (src/operators/NonlocalProjector.cpp:165-181): per image, ndc grid points,
// Chi column-major (ndc x nproj); Gamma per (atom, projector).
int ref_nl_tables(int* img_atom, int* img_ndc, double* img_shift, double* img_coords, int* gpos,
                  double* chi, double* gamma, double* rc) {
    if (!g || !g->has_vnl) return -1;
    const auto& inf = g->nloc[0];
    const auto& psd = g->crystal->types()[0].psd();
    int nproj = psd.nproj_per_atom();
    long off = 0;
    for (int i = 0; i < inf.n_atom; ++i) {
        img_atom[i] = inf.atom_index[i];
        img_ndc[i] = inf.ndc[i];
        img_shift[3 * i] = inf.image_shift[i].x;
        img_shift[3 * i + 1] = inf.image_shift[i].y;
        img_shift[3 * i + 2] = inf.image_shift[i].z;
        img_coords[3 * i] = inf.coords[i].x;
        img_coords[3 * i + 1] = inf.coords[i].y;
        img_coords[3 * i + 2] = inf.coords[i].z;
        int ndc = inf.ndc[i];
        for (int gi = 0; gi < ndc; ++gi) gpos[off + gi] = inf.grid_pos[i][gi];
        const auto& C = g->vnl.Chi_[0][i];
        for (int jp = 0; jp < nproj; ++jp)
            for (int gi = 0; gi < ndc; ++gi) chi[off * nproj + (long)jp * ndc + gi] = C(gi, jp);
        off += ndc;
    }
    int na = g->crystal->n_atom_total();
    int c = 0;
    for (int a = 0; a < na; ++a)
        for (int l = 0; l <= psd.lmax(); ++l) {
            if (l == psd.lloc()) continue;
            for (int p = 0; p < psd.ppl()[l]; ++p)
                for (int m = -l; m <= l; ++m) gamma[c++] = psd.Gamma()[l][p];
        }
    if (rc) {
        double r = 0;
        for (double x : psd.rc()) r = std::max(r, x);
        *rc = r;
    }
    return 0;
}

// Hamiltonian::apply (src/operators/Hamiltonian.cpp:22,64): y = H psi + c psi.
int ref_h_apply(const double* psi, const double* veff, double* y, int ncol, double c) {
    if (!g) return -1;
    return guarded([&] { g->H.apply(psi, veff, y, ncol, c); });
}

// Hamiltonian::apply_kpt (src/operators/Hamiltonian.cpp:30,81); psi, y interleaved complex.
int ref_h_apply_kpt(const double* psi, const double* veff, double* y, int ncol, const double* kpt,
                    double c) {
    if (!g) return -1;
    return guarded([&] {
        Vec3 k(kpt[0], kpt[1], kpt[2]);
        if (g->has_vnl) g->vnl.set_kpoint(k);
        g->H.apply_kpt(reinterpret_cast<const Complex*>(psi), veff, reinterpret_cast<Complex*>(y), ncol, k,
                       g->lattice.lengths(), c);
    });
}

// NonlocalProjector::apply (src/operators/NonlocalProjector.cpp:121): hpsi += Vnl psi.
int ref_nl_apply(const double* psi, double* hpsi, int ncol) {
    if (!g || !g->has_vnl) return -1;
    return guarded([&] { g->vnl.apply(psi, hpsi, ncol, g->grid.dV()); });
}

int ref_nl_apply_kpt(const double* psi, double* hpsi, int ncol, const double* kpt) {
    if (!g || !g->has_vnl) return -1;
    return guarded([&] {
        g->vnl.set_kpoint(Vec3(kpt[0], kpt[1], kpt[2]));
        g->vnl.apply_kpt(reinterpret_cast<const Complex*>(psi), reinterpret_cast<Complex*>(hpsi), ncol,
                         g->grid.dV());
    });
}

// EigenSolver::chebyshev_filter_impl (src/solvers/EigenSolver.cpp:559-619).
int ref_chebyshev_filter(const double* X, double* Y, const double* veff, int ncol, double lc, double emin,
                         double emax, int degree) {
    if (!g) return -1;
    return guarded([&] {
        g->es.chebyshev_filter_impl<double>(X, Y, veff, g->domain.Nd_d(), ncol, lc, emin, emax, degree);
    });
}

int ref_chebyshev_filter_kpt(const double* X, double* Y, const double* veff, int ncol, double lc,
                             double emin, double emax, int degree, const double* kpt) {
    if (!g) return -1;
    return guarded([&] {
        Vec3 k(kpt[0], kpt[1], kpt[2]);
        if (g->has_vnl) g->vnl.set_kpoint(k);
        g->es.chebyshev_filter_impl<Complex>(reinterpret_cast<const Complex*>(X), reinterpret_cast<Complex*>(Y),
                                             veff, g->domain.Nd_d(), ncol, lc, emin, emax, degree, k,
                                             g->lattice.lengths());
    });
}

// EigenSolver::solve (src/solvers/EigenSolver.cpp:739-829).
int ref_solve(double* psi, double* eig, const double* veff, int nband, double lc, double emin, double emax,
              int degree) {
    if (!g) return -1;
    return guarded([&] { g->es.solve(psi, eig, veff, g->domain.Nd_d(), nband, lc, emin, emax, degree); });
}

// EigenSolver::solve_kpt (src/solvers/EigenSolver.cpp:831-842).
int ref_solve_kpt(double* psi, double* eig, const double* veff, int nband, double lc, double emin,
                  double emax, int degree, const double* kpt) {
    if (!g) return -1;
    return guarded([&] {
        Vec3 k(kpt[0], kpt[1], kpt[2]);
        if (g->has_vnl) g->vnl.set_kpoint(k);
        g->es.solve_kpt(reinterpret_cast<Complex*>(psi), eig, veff, g->domain.Nd_d(), nband, lc, emin, emax, k,
                        g->lattice.lengths(), degree);
    });
}

double ref_lambda_cutoff() { return g ? g->es.lambda_cutoff() : 0.0; }

// Individual Rayleigh-Ritz steps (src/solvers/EigenSolver.cpp:622-681).
int ref_orthogonalize(double* X, int ncol) {
    if (!g) return -1;
    return guarded([&] { g->es.orthogonalize_impl<double>(X, g->domain.Nd_d(), ncol, g->grid.dV()); });
}
int ref_project(const double* X, const double* veff, double* Hs, int ncol) {
    if (!g) return -1;
    return guarded([&] {
        g->es.project_hamiltonian_impl<double>(X, veff, Hs, g->domain.Nd_d(), ncol, g->grid.dV());
    });
}
int ref_diag(double* Hs, double* eig, int n) {
    if (!g) return -1;
    return guarded([&] { g->es.diag_subspace_impl<double>(Hs, eig, n); });
}
int ref_rotate(double* X, const double* Q, int ncol) {
    if (!g) return -1;
    return guarded([&] { g->es.rotate_orbitals_impl<double>(X, Q, g->domain.Nd_d(), ncol); });
}

// EigenSolver::lanczos_bounds (src/solvers/EigenSolver.cpp:724-732 -> Lanczos.hpp:92-200).
int ref_lanczos(const double* veff, double* emin, double* emax, double tol, int maxit) {
    if (!g) return -1;
    return guarded([&] { g->es.lanczos_bounds(veff, g->domain.Nd_d(), *emin, *emax, tol, maxit); });
}
int ref_lanczos_kpt(const double* veff, double* emin, double* emax, double tol, int maxit, const double* kpt) {
    if (!g) return -1;
    return guarded([&] {
        Vec3 k(kpt[0], kpt[1], kpt[2]);
        if (g->has_vnl) g->vnl.set_kpoint(k);
        g->es.lanczos_bounds_kpt(veff, g->domain.Nd_d(), k, g->lattice.lengths(), *emin, *emax, tol, maxit);
    });
}

// Occupation::find_fermi_level (src/electronic/Occupation.cpp:48-84) and the smearing functions.
double ref_fermi_level(const double* eigs, const double* w, int n, double Ne, double beta, int fermi_dirac) {
    std::vector<double> e(eigs, eigs + n), ww(w, w + n);
    double ef = 0.0;
    int rc = guarded([&] {
        ef = lynx::Occupation::find_fermi_level(
            e, ww, Ne, beta, fermi_dirac ? lynx::SmearingType::FermiDirac : lynx::SmearingType::GaussianSmearing);
    });
    return rc == 0 ? ef : NAN;
}
double ref_smearing(double x, double beta, int fermi_dirac) {
    return lynx::Occupation::smearing_function(
        x, beta, fermi_dirac ? lynx::SmearingType::FermiDirac : lynx::SmearingType::GaussianSmearing);
}

// KPoints::generate (src/core/KPoints.cpp:8-80) on the current lattice.
int ref_kpoints(int kx, int ky, int kz, const double* shift, double* kcart, double* kred, double* w, int maxk) {
    if (!g) return -1;
    lynx::KPoints kp;
    kp.generate(kx, ky, kz, Vec3(shift[0], shift[1], shift[2]), g->lattice);
    int n = kp.Nkpts();
    for (int i = 0; i < n && i < maxk; ++i) {
        kcart[3 * i] = kp.kpts_cart()[i].x;
        kcart[3 * i + 1] = kp.kpts_cart()[i].y;
        kcart[3 * i + 2] = kp.kpts_cart()[i].z;
        kred[3 * i] = kp.kpts_red()[i].x;
        kred[3 * i + 1] = kp.kpts_red()[i].y;
        kred[3 * i + 2] = kp.kpts_red()[i].z;
        w[i] = kp.weights()[i];
    }
    return n;
}

// ---------------------------------------------------------------------------
// Nonlocal forces, kinetic / nonlocal stress and the electron density of given orbitals,
// by the reference's own Forces::compute_nonlocal_cpu (src/physics/Forces.cpp:509-797),
// Stress::compute_nonlocal_kinetic_cpu (src/physics/Stress.cpp:1041-1784) and
// ElectronDensity::compute (src/electronic/ElectronDensity.cpp:55-172), for one spin channel
// (Nspin = 1, so occfac = 2) and one k-point of weight wk (psi complex when is_kpt, at the
// Cartesian k-point kpt).  The objects those routines read from the LynxContext singleton
// (gradient, halo, domain, grid, communicators, k-points) are assembled here directly.
// ---------------------------------------------------------------------------
namespace {
// One Wavefunction holding psi (Nd x nband, column-major) and the occupations.
void fill_wfn(lynx::Wavefunction& w, const double* psi, const double* occ, int nband, bool is_kpt) {
    const int nd = g->domain.Nd_d();
    w.allocate(nd, nband, 1, 1, is_kpt);
    if (is_kpt) {
        std::memcpy(w.psi_kpt(0, 0).data(), psi, sizeof(Complex) * (size_t)nd * nband);
    } else {
        std::memcpy(w.psi(0, 0).data(), psi, sizeof(double) * (size_t)nd * nband);
    }
    std::memcpy(w.occupations(0, 0).data(), occ, sizeof(double) * nband);
}
// A LynxContext with the pieces Forces::compute_nonlocal_cpu reads (one rank, one spin, one
// k-point).  Its constructor is private (reachable through the harness's access defines); it is
// never destroyed, as the reference's destructor finalises MPI and is not linked here.
lynx::LynxContext* make_context(int nband, const double* kpt) {
    auto* c = new lynx::LynxContext();
    c->lattice_.reset(new lynx::Lattice(g->lattice));
    c->grid_.reset(new lynx::FDGrid(g->grid));
    c->stencil_.reset(new lynx::FDStencil(g->stencil));
    lynx::ParallelParams pp;
    c->parallel_.reset(new lynx::Parallelization(MPI_COMM_WORLD, pp, g->grid, 1, 1, nband));
    c->parallel_->domain_ = g->domain;
    c->halo_.reset(new lynx::HaloExchange(g->domain, g->stencil.FDn()));
    c->gradient_.reset(new lynx::Gradient(g->stencil, g->domain));
    c->kpoints_.reset(new lynx::KPoints());
    c->kpoints_->kpts_cart_.assign(1, kpt ? Vec3(kpt[0], kpt[1], kpt[2]) : Vec3(0, 0, 0));
    c->kpoints_->weights_.assign(1, 1.0);
    c->scf_bandcomm_ = &c->parallel_->bandcomm();
    return c;
}
}  // namespace

// force: 3 * n_atom doubles (atom-major), the reference's f_nloc_.
int ref_nonlocal_force(const double* psi, const double* occ, int nband, int is_kpt, const double* kpt, double wk,
                       double* force) {
    if (!g || !g->has_vnl) return -1;
    return guarded([&] {
        if (is_kpt) g->vnl.set_kpoint(Vec3(kpt[0], kpt[1], kpt[2]));
        lynx::Wavefunction w;
        fill_wfn(w, psi, occ, nband, is_kpt != 0);
        lynx::Forces f;
        f.ctx_ = make_context(nband, is_kpt ? kpt : nullptr);
        f.compute_nonlocal_cpu(w, *g->crystal, g->nloc, g->vnl, std::vector<double>(1, wk));
        std::memcpy(force, f.f_nloc_.data(), sizeof(double) * f.f_nloc_.size());
    });
}

// stress_k, stress_nl: 6 doubles each (Voigt xx, xy, xz, yy, yz, zz), before the division by the
// cell measure (the reference divides by Stress::cell_measure_, set to 1 here).
int ref_kinetic_nonlocal_stress(const double* psi, const double* occ, int nband, int is_kpt, const double* kpt,
                                double wk, double* stress_k, double* stress_nl) {
    if (!g) return -1;
    return guarded([&] {
        if (is_kpt && g->has_vnl) g->vnl.set_kpoint(Vec3(kpt[0], kpt[1], kpt[2]));
        lynx::Wavefunction w;
        fill_wfn(w, psi, occ, nband, is_kpt != 0);
        lynx::LynxContext* c = make_context(nband, is_kpt ? kpt : nullptr);
        lynx::Stress st;
        st.cell_measure_ = 1.0;
        lynx::Crystal empty_crystal;
        const lynx::Crystal& cr = g->has_vnl ? *g->crystal : empty_crystal;
        std::vector<lynx::AtomNlocInfluence> no_nloc;
        st.compute_nonlocal_kinetic_cpu(w, cr, g->has_vnl ? g->nloc : no_nloc, g->vnl, c->gradient(), c->halo(),
                                        c->domain(), c->grid(), std::vector<double>(1, wk), c->scf_bandcomm(),
                                        c->kpt_bridge(), c->spin_bridge(), &c->kpoints(), 0, 0);
        std::memcpy(stress_k, st.stress_k_.data(), 6 * sizeof(double));
        std::memcpy(stress_nl, st.stress_nl_.data(), 6 * sizeof(double));
    });
}

// rho: Nd doubles, rho = sum_n 2 wk occ[n] |psi_n|^2 (Nspin = 1).
int ref_density(const double* psi, const double* occ, int nband, int is_kpt, double wk, double* rho) {
    if (!g) return -1;
    return guarded([&] {
        lynx::Wavefunction w;
        fill_wfn(w, psi, occ, nband, is_kpt != 0);
        lynx::LynxContext* c = make_context(nband, nullptr);
        lynx::ElectronDensity d;
        d.allocate(g->domain.Nd_d(), 1);
        d.compute(w, std::vector<double>(1, wk), g->grid.dV(), c->scf_bandcomm(), c->kpt_bridge(), 1, 0, nullptr, 0,
                  0);
        std::memcpy(rho, d.rho_total().data(), sizeof(double) * g->domain.Nd_d());
    });
}

// Wavefunction::randomize convention (src/electronic/Wavefunction.cpp:53-63).
void ref_randomize(double* x, long n, unsigned seed) {
    std::srand(seed);
    for (long i = 0; i < n; ++i) x[i] = -0.5 + 1.0 * ((double)std::rand() / RAND_MAX);
}

// PoissonSolver::solve on the set-up grid (src/solvers/PoissonSolver.cpp:17-159): -Lap phi = rhs
// from the start phi; *iters receives the AAR step count.
int ref_poisson(const double* rhs, double* phi, double tol, int* iters) {
    return guarded([&] {
        lynx::Laplacian lap(g->stencil, g->domain);
        lynx::PoissonSolver ps;
        ps.setup(lap, g->stencil, g->domain, g->grid, g->halo);
        *iters = ps.solve(rhs, phi, tol);
    });
}

// Gradient::apply along direction dir of one field, ghosts from HaloExchange::execute
// (src/operators/Gradient.cpp:17-62).
int ref_gradient(const double* x, double* y, int dir) {
    return guarded([&] {
        lynx::Gradient grad(g->stencil, g->domain);
        std::vector<double> xe(g->halo.nd_ex(), 0.0);
        g->halo.execute(x, xe.data(), 1);
        grad.apply(xe.data(), y, dir, 1);
    });
}

int ref_set_threads(int n) {
    omp_set_num_threads(n);
    return omp_get_max_threads();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Link-time stand-ins for symbols the reference Hamiltonian references on code
// paths the eigensolver never takes here (hybrid EXX is never set up, mGGA
// vtau is never set).  They throw if ever reached.
// ---------------------------------------------------------------------------
namespace lynx {
void ExactExchange::apply_Vx(const double*, int, int, int, double*, int, int) const {
    throw std::runtime_error("EXX not available in the oracle harness");
}
void ExactExchange::apply_Vx_kpt(const Complex*, int, int, int, Complex*, int, int, int) const {
    throw std::runtime_error("EXX not available in the oracle harness");
}
}  // namespace lynx
