// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C-ABI shim over the *reference* waveDG library (compiled from its own
// sources by oracle/Makefile into oracle/_ref/).  It calls only the
// reference's public API and exists so that the tests can pin the oracle and
// the GPU path against the reference's own arithmetic, and so that bench.py
// can time the reference's CPU code as the baseline.  Nothing in the product
// path links or loads this file.
//
// Two operators are not available verbatim from the reference and are
// composed here from its public parts exactly as WaveBC::action composes them
// (source/WaveEquation.cpp:190-215):
//   * code 0, absorbing (outflow): wavedg/WaveEquation.hpp:77-84 assigns
//     v_ext[0] from v_ext[1], v_ext[2] *before* those are computed, so the
//     verbatim code reads the previous node's values (and uninitialised stack
//     at the first node).  The composed operator evaluates the same three
//     statements in dependency order: velocity first, then p_ext = n . u_ext.
//   * code 2, Dirichlet p = 0: not implemented for 2D by the reference
//     (WaveBC accepts 0/1 only, source/WaveEquation.cpp:80-81); the mirror
//     state p_ext = -p, u_ext = u is fed through the same boundary flux.
// Code 1 (reflecting) uses dg::reflect_2d (wavedg/WaveEquation.hpp:64-69).

#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

#include "wavedg.hpp"

using namespace dg;

namespace
{
    // wave system as a constant-coefficient conservation law; the same table
    // the reference builds in source/WaveEquation.cpp:10-18.
    const double kWaveA[] = {
        0.0, 1.0, 0.0,
        1.0, 0.0, 0.0,
        0.0, 0.0, 0.0,

        0.0, 0.0, 1.0,
        0.0, 0.0, 0.0,
        1.0, 0.0, 0.0};

    FaceType face_type(int t) { return t == 0 ? FaceType::INTERIOR : FaceType::BOUNDARY; }

    void exterior_state(int code, double v_ext[3], const double v_int[3], const double n[2])
    {
        if (code == 1)
        {
            reflect_2d(v_ext, v_int, n);
        }
        else if (code == 0)
        {
            const double outgoing = v_int[0] + n[0] * v_int[1] + n[1] * v_int[2];
            const double tangential = n[1] * v_int[1] - n[0] * v_int[2];
            v_ext[1] = n[1] * tangential + 0.5 * n[0] * outgoing;
            v_ext[2] = -n[0] * tangential + 0.5 * n[1] * outgoing;
            v_ext[0] = n[0] * v_ext[1] + n[1] * v_ext[2];
        }
        else
        {
            v_ext[0] = -v_int[0];
            v_ext[1] = v_int[1];
            v_ext[2] = v_int[2];
        }
    }

    struct RefMesh
    {
        Mesh2D mesh;
        explicit RefMesh(Mesh2D &&m) : mesh(std::move(m)) {}
    };

    // boundary operator with the exterior states above, built from the
    // reference's boundary prolongator, FaceVector and EdgeFlux<true>.
    struct ComposedBC : public Operator
    {
        const int nB, n;
        std::unique_ptr<FaceProlongator> prol;
        std::unique_ptr<Operator> flx; // EdgeFlux<true> or, exact quadrature, EdgeFlux<false>
        const double *normals;
        std::vector<int> bc;
        mutable FaceVector uB;

        ComposedBC(const Mesh2D &mesh, const QuadratureRule *basis, const int *codes, bool approx = true)
            : nB(mesh.n_edges(FaceType::BOUNDARY)), n(basis->n),
              prol(make_face_prolongator(mesh, basis, FaceType::BOUNDARY)),
              flx(approx ? static_cast<Operator *>(new EdgeFlux<true>(3, mesh, FaceType::BOUNDARY, basis, kWaveA, true))
                         : static_cast<Operator *>(new EdgeFlux<false>(3, mesh, FaceType::BOUNDARY, basis, kWaveA,
                                                                      true, -1.0, -0.5, nullptr))),
              normals(mesh.edge_metrics(basis, FaceType::BOUNDARY).normals()),
              bc(codes, codes + mesh.n_edges(FaceType::BOUNDARY)),
              uB(3, mesh, FaceType::BOUNDARY, basis) {}

        void exterior(double *uB_) const
        {
            auto U = reshape(uB_, n, 3, 2, nB);
            auto N = reshape(normals, 2, n, nB);
            double vi[3], ve[3];
            for (int e = 0; e < nB; ++e)
                for (int i = 0; i < n; ++i)
                {
                    for (int d = 0; d < 3; ++d)
                        vi[d] = U(i, d, 0, e);
                    exterior_state(bc[e], ve, vi, &N(0, i, e));
                    for (int d = 0; d < 3; ++d)
                        U(i, d, 1, e) = ve[d];
                }
        }

        void action(const double *u, double *du) const override
        {
            prol->action(3, u, uB);
            exterior(uB);
            flx->action(uB, uB);
            prol->t(3, uB, du);
        }
        void action(int, const double *u, double *du) const override { action(u, du); }
    };

    struct RefOp
    {
        static constexpr bool approx = true;
        const Mesh2D &mesh;
        const QuadratureRule *basis;
        const int n, nel, ndof;
        std::vector<int> codes;
        bool all_reflect;
        WaveEquation a;
        std::unique_ptr<WaveBC> native_bc; // only constructible for codes 0/1
        ComposedBC bc;
        MassMatrix<true> m;
        // stand-alone component operators, built on first use
        mutable std::unique_ptr<Div<true>> div_;
        mutable std::unique_ptr<FaceProlongator> prolI_, prolB_;
        mutable std::unique_ptr<EdgeFlux<true>> flxI_, flxB_;

        RefOp(const Mesh2D &mesh_, int n_colloc, const int *bc_)
            : mesh(mesh_), basis(QuadratureRule::quadrature_rule(n_colloc, QuadratureRule::GaussLobatto)),
              n(n_colloc), nel(mesh_.n_elem()), ndof(3 * n_colloc * n_colloc * mesh_.n_elem()),
              codes(bc_, bc_ + mesh_.n_edges(FaceType::BOUNDARY)),
              all_reflect(true),
              a(mesh_, basis, true),
              bc(mesh_, basis, bc_),
              m(mesh_, basis)
        {
            bool only01 = true;
            for (int c : codes)
            {
                all_reflect = all_reflect && (c == 1);
                only01 = only01 && (c == 0 || c == 1);
            }
            if (only01)
                native_bc.reset(new WaveBC(mesh_, codes.data(), basis, true));
        }

        const Div<true> &div() const
        {
            if (!div_)
                div_.reset(new Div<true>(3, mesh, basis, kWaveA, true));
            return *div_;
        }
        const FaceProlongator &prol(int type) const
        {
            auto &p = (type == 0) ? prolI_ : prolB_;
            if (!p)
                p = make_face_prolongator(mesh, basis, face_type(type));
            return *p;
        }
        const EdgeFlux<true> &flx(int type) const
        {
            auto &f = (type == 0) ? flxI_ : flxB_;
            if (!f)
                f.reset(new EdgeFlux<true>(3, mesh, face_type(type), basis, kWaveA, true));
            return *f;
        }

        // time derivative of the examples: M^{-1} (A u + B u + s F)
        void rhs(const double *u, double *du, const double *F, double s) const
        {
            for (int i = 0; i < ndof; ++i)
                du[i] = 0.0;
            a.action(u, du);
            bc.action(u, du);
            if (F)
                for (int i = 0; i < ndof; ++i)
                    du[i] += F[i] * s;
            m.inv(3, du);
        }
    };

    // The same system with approx_quad = false: WaveEquation(mesh, basis, false)
    // (source/WaveEquation.cpp:5-30: Div<false>, EdgeFlux<false> with the default rules),
    // the composed boundary operator over EdgeFlux<false> (WaveBC with approx_quad = false,
    // :70-105) and MassMatrix<false> (source/MassMatrix.cpp:84-230).
    struct RefOpQ
    {
        static constexpr bool approx = false;
        const Mesh2D &mesh;
        const QuadratureRule *basis;
        const int n, nel, ndof;
        std::vector<int> codes;
        bool all_reflect = true;
        WaveEquation a;
        ComposedBC bc;
        MassMatrix<false> m;
        Div<false> div;
        EdgeFlux<false> flxI, flxB;

        RefOpQ(const Mesh2D &mesh_, int n_colloc, const int *bc_)
            : mesh(mesh_), basis(QuadratureRule::quadrature_rule(n_colloc, QuadratureRule::GaussLobatto)),
              n(n_colloc), nel(mesh_.n_elem()), ndof(3 * n_colloc * n_colloc * mesh_.n_elem()),
              codes(bc_, bc_ + mesh_.n_edges(FaceType::BOUNDARY)),
              a(mesh_, basis, false),
              bc(mesh_, basis, bc_, false),
              m(mesh_, basis),
              div(3, mesh_, basis, kWaveA, true, nullptr),
              flxI(3, mesh_, FaceType::INTERIOR, basis, kWaveA, true, -1.0, -0.5, nullptr),
              flxB(3, mesh_, FaceType::BOUNDARY, basis, kWaveA, true, -1.0, -0.5, nullptr)
        {
            for (int c : codes)
                all_reflect = all_reflect && (c == 1);
        }

        void rhs(const double *u, double *du, const double *F = nullptr, double s = 0.0) const
        {
            for (int i = 0; i < ndof; ++i)
                du[i] = 0.0;
            a.action(u, du);
            bc.action(u, du);
            if (F)
                for (int i = 0; i < ndof; ++i)
                    du[i] += F[i] * s;
            m.inv(3, du);
        }
    };

    // Advection<true> and AdvectionHomogeneousBC<true> (wavedg/Advection.hpp) with constant
    // coefficients a (n_var, n_var, 2), and MassMatrix<true>
    struct RefOpA
    {
        const Mesh2D &mesh;
        const QuadratureRule *basis;
        const int nv, ndof;
        std::vector<double> a;
        Advection<true> adv;
        AdvectionHomogeneousBC<true> bc;
        MassMatrix<true> m;

        RefOpA(const Mesh2D &mesh_, int n_colloc, int nv_, const double *a_)
            : mesh(mesh_), basis(QuadratureRule::quadrature_rule(n_colloc, QuadratureRule::GaussLobatto)), nv(nv_),
              ndof(nv_ * n_colloc * n_colloc * mesh_.n_elem()), a(a_, a_ + 2 * nv_ * nv_),
              adv(nv_, mesh_, basis, a.data(), true), bc(nv_, mesh_, basis, a.data(), true), m(mesh_, basis)
        {
        }
        void rhs(const double *u, double *du) const
        {
            for (int i = 0; i < ndof; ++i)
                du[i] = 0.0;
            adv.action(u, du);
            bc.action(u, du);
            m.inv(nv, du);
        }
    };

    // Advection<AQ> and AdvectionHomogeneousBC<AQ> with a spatially varying coefficient
    // a(n_var, n_var, 2, n, n, n_elem) (constant_coefficient = false, wavedg/Advection.hpp:59-273)
    // and MassMatrix<AQ>, on a Gauss-Lobatto or Gauss-Legendre basis
    struct RefOpVBase
    {
        int nv = 0, ndof = 0;
        virtual ~RefOpVBase() = default;
        virtual void action(const double *u, double *du) const = 0;
        virtual void bc_action(const double *u, double *du) const = 0;
        virtual void inv(double *du) const = 0;
        void rhs(const double *u, double *du) const
        {
            for (int i = 0; i < ndof; ++i)
                du[i] = 0.0;
            action(u, du);
            bc_action(u, du);
            inv(du);
        }
    };
    template <bool AQ>
    struct RefOpV : RefOpVBase
    {
        const QuadratureRule *basis;
        std::vector<double> a;
        Advection<AQ> adv;
        AdvectionHomogeneousBC<AQ> bc;
        MassMatrix<AQ> m;

        RefOpV(const Mesh2D &mesh, int n_colloc, int nv_, const double *a_, QuadratureRule::QuadratureType type)
            : basis(QuadratureRule::quadrature_rule(n_colloc, type)),
              a(a_, a_ + (size_t)2 * nv_ * nv_ * n_colloc * n_colloc * mesh.n_elem()),
              adv(nv_, mesh, basis, a.data(), false), bc(nv_, mesh, basis, a.data(), false), m(mesh, basis)
        {
            nv = nv_;
            ndof = nv_ * n_colloc * n_colloc * mesh.n_elem();
        }
        void action(const double *u, double *du) const override { adv.action(u, du); }
        void bc_action(const double *u, double *du) const override { bc.action(u, du); }
        void inv(double *du) const override { m.inv(nv, du); }
    };

    // The compressible Euler system of examples/cl2d.cpp (gamma = 1.4): its physical flux,
    // wave speed and local Lax-Friedrichs numerical flux, as that example defines them
    // (cl2d.cpp:67-126), for the reference's nonlinear operators below.
    constexpr double kGamma = 1.4;
    void euler_flux(const double *, const double q[4], double fg[8])
    {
        const double rho = q[0], u = q[1] / q[0], v = q[2] / q[0], E = q[3];
        const double p = (kGamma - 1.0) * (E - 0.5 * rho * (u * u + v * v));
        fg[0] = rho * u;
        fg[1] = rho * u * u + p;
        fg[2] = rho * u * v;
        fg[3] = u * (E + p);
        fg[4] = rho * v;
        fg[5] = rho * u * v;
        fg[6] = rho * v * v + p;
        fg[7] = v * (E + p);
    }
    double euler_speed(const double q[4])
    {
        const double rho = q[0], u = q[1] / q[0], v = q[2] / q[0], E = q[3];
        const double p = (kGamma - 1.0) * (E - 0.5 * rho * (u * u + v * v));
        return std::hypot(u, v) + std::sqrt(kGamma * p / rho);
    }
    void euler_llf(const double *x, const double nrm[2], const double qL[4], const double qR[4], double fh[4])
    {
        double fL[8], fR[8];
        euler_flux(x, qL, fL);
        euler_flux(x, qR, fR);
        const double c = std::max(euler_speed(qL), euler_speed(qR));
        for (int d = 0; d < 4; ++d)
            fh[d] = 0.5 * nrm[0] * (fL[d] + fR[d]) + 0.5 * nrm[1] * (fL[4 + d] + fR[4 + d]) + 0.5 * c * (qL[d] - qR[d]);
    }

    // DivF2D<true>, EdgeFluxF2D<true> (interior and boundary), the Lobatto prolongators and
    // MassMatrix<true>, composed into the time derivative of examples/cl2d.cpp:171-220 with
    // approx_quad = true: exterior boundary state = interior state.
    struct RefOpE
    {
        static constexpr int nv = 4;
        const Mesh2D &mesh;
        const QuadratureRule *basis;
        const int n, ndof, nI, nB;
        DivF2D<true> div;
        EdgeFluxF2D<true> flxI, flxB;
        std::unique_ptr<FaceProlongator> prolI, prolB;
        MassMatrix<true> m;
        mutable std::vector<double> uI, uB;

        RefOpE(const Mesh2D &mesh_, int n_colloc)
            : mesh(mesh_), basis(QuadratureRule::quadrature_rule(n_colloc, QuadratureRule::GaussLobatto)), n(n_colloc),
              ndof(nv * n_colloc * n_colloc * mesh_.n_elem()), nI(mesh_.n_edges(FaceType::INTERIOR)),
              nB(mesh_.n_edges(FaceType::BOUNDARY)), div(mesh_, basis), flxI(mesh_, FaceType::INTERIOR, basis),
              flxB(mesh_, FaceType::BOUNDARY, basis), prolI(make_face_prolongator(mesh_, basis, FaceType::INTERIOR)),
              prolB(make_face_prolongator(mesh_, basis, FaceType::BOUNDARY)), m(mesh_, basis),
              uI((size_t)n_colloc * nv * 2 * nI), uB((size_t)n_colloc * nv * 2 * nB)
        {
        }
        void flux(int type, const double *ub, double *fb) const
        {
            (type == 0 ? flxI : flxB).action(nv, euler_llf, ub, fb);
        }
        void rhs(const double *u, double *dudt) const
        {
            for (int i = 0; i < ndof; ++i)
                dudt[i] = 0.0;
            div.action(nv, euler_flux, u, dudt);
            prolI->action(nv, u, uI.data());
            flxI.action(nv, euler_llf, uI.data(), uI.data());
            for (double &x : uI)
                x *= -1;
            prolI->t(nv, uI.data(), dudt);
            prolB->action(nv, u, uB.data());
            for (int e = 0; e < nB; ++e)
                for (int d = 0; d < nv; ++d)
                    for (int i = 0; i < n; ++i)
                        uB[i + n * (d + nv * (1 + 2 * (size_t)e))] = uB[i + n * (d + nv * (0 + 2 * (size_t)e))];
            flxB.action(nv, euler_llf, uB.data(), uB.data());
            for (double &x : uB)
                x *= -1;
            prolB->t(nv, uB.data(), dudt);
            m.inv(nv, dudt);
        }
    };

    // The same composition with approx_quad = false, as examples/cl2d.cpp ships: DivF2D<false>,
    // EdgeFluxF2D<false> (their default 2n-point rules) and MassMatrix<false>.
    struct RefOpEQ
    {
        static constexpr int nv = 4;
        const Mesh2D &mesh;
        const QuadratureRule *basis;
        const int n, ndof, nI, nB;
        DivF2D<false> div;
        EdgeFluxF2D<false> flxI, flxB;
        std::unique_ptr<FaceProlongator> prolI, prolB;
        MassMatrix<false> m;
        mutable std::vector<double> uI, uB;

        RefOpEQ(const Mesh2D &mesh_, int n_colloc)
            : mesh(mesh_), basis(QuadratureRule::quadrature_rule(n_colloc, QuadratureRule::GaussLobatto)), n(n_colloc),
              ndof(nv * n_colloc * n_colloc * mesh_.n_elem()), nI(mesh_.n_edges(FaceType::INTERIOR)),
              nB(mesh_.n_edges(FaceType::BOUNDARY)), div(mesh_, basis), flxI(mesh_, FaceType::INTERIOR, basis),
              flxB(mesh_, FaceType::BOUNDARY, basis), prolI(make_face_prolongator(mesh_, basis, FaceType::INTERIOR)),
              prolB(make_face_prolongator(mesh_, basis, FaceType::BOUNDARY)), m(mesh_, basis),
              uI((size_t)n_colloc * nv * 2 * nI), uB((size_t)n_colloc * nv * 2 * nB)
        {
        }
        void flux(int type, const double *ub, double *fb) const
        {
            (type == 0 ? flxI : flxB).action(nv, euler_llf, ub, fb);
        }
        void rhs(const double *u, double *dudt) const
        {
            for (int i = 0; i < ndof; ++i)
                dudt[i] = 0.0;
            div.action(nv, euler_flux, u, dudt);
            prolI->action(nv, u, uI.data());
            flxI.action(nv, euler_llf, uI.data(), uI.data());
            for (double &x : uI)
                x *= -1;
            prolI->t(nv, uI.data(), dudt);
            prolB->action(nv, u, uB.data());
            for (int e = 0; e < nB; ++e)
                for (int d = 0; d < nv; ++d)
                    for (int i = 0; i < n; ++i)
                        uB[i + n * (d + nv * (1 + 2 * (size_t)e))] = uB[i + n * (d + nv * (0 + 2 * (size_t)e))];
            flxB.action(nv, euler_llf, uB.data(), uB.data());
            for (double &x : uB)
                x *= -1;
            prolB->t(nv, uB.data(), dudt);
            m.inv(nv, dudt);
        }
    };

    // WaveHoltz restated over RefOp so that the composed boundary operator can
    // be used (the reference class hard-wires WaveBC).  Loop structure, time
    // accumulation and filter weights follow source/WaveHoltz.cpp:5-145; with
    // all-reflecting boundaries the reference class itself is used instead.
    template <class O>
    struct RefWHT
    {
        const O &op;
        const double omega;
        double T, dt;
        int nt;
        std::unique_ptr<WaveHoltz> native;
        ode::RungeKutta4 rk;
        mutable std::vector<double> p;

        RefWHT(const O &op_, double omega_) : op(op_), omega(omega_), rk(op_.ndof), p(op_.ndof)
        {
            T = 2.0 * M_PI / omega;
            double h = op.mesh.min_h();
            double pp = op.basis->n;
            dt = 0.5 * h / (pp * pp);
            nt = std::ceil(T / dt);
            dt = T / nt;
            if (op.all_reflect)
                native.reset(new WaveHoltz(omega, op.mesh, op.basis, op.codes.data(), O::approx));
        }

        double K(double t) const { return omega / M_PI * (std::cos(omega * t) - 0.25); }

        void pi0(double *u, const double *F) const
        {
            if (native)
            {
                native->pi0(u, F);
                return;
            }
            const int ndof = op.ndof;
            auto f = [this, F](double *vt, const double t, const double *v)
            { op.rhs(v, vt, F, -1.0 / omega * std::sin(omega * t)); };
            for (int i = 0; i < ndof; ++i)
                p[i] = u[i] = 0.0;
            double t = 0.0;
            for (int it = 1; it <= nt; ++it)
            {
                rk.step(dt, f, t, p.data());
                const double c = ((it == nt) ? 0.5 : 1.0) * dt * K(t);
                for (int i = 0; i < ndof; ++i)
                    u[i] += c * p[i];
            }
        }

        void S(double *u) const
        {
            if (native)
            {
                native->S(u);
                return;
            }
            const int ndof = op.ndof;
            auto f = [this](double *vt, const double, const double *v)
            { op.rhs(v, vt, nullptr, 0.0); };
            for (int i = 0; i < ndof; ++i)
            {
                p[i] = u[i];
                u[i] *= 0.5 * dt * K(0.0);
            }
            double t = 0.0;
            for (int it = 1; it <= nt; ++it)
            {
                rk.step(dt, f, t, p.data());
                const double c = ((it == nt) ? 0.5 : 1.0) * dt * K(t);
                for (int i = 0; i < ndof; ++i)
                    u[i] += c * p[i];
            }
        }

        void postprocess(double *H, const double *U) const
        {
            if (native)
            {
                native->postprocess(H, U);
                return;
            }
            const int npts = op.ndof / 3;
            op.rhs(U, p.data(), nullptr, 0.0);
            for (int i = 0; i < npts; ++i)
            {
                H[2 * i] = U[3 * i];
                H[2 * i + 1] = -1.0 / omega * p[3 * i];
            }
        }
    };
    using RefWH = RefWHT<RefOp>;
    using RefWHQ = RefWHT<RefOpQ>;
} // namespace

namespace
{
    // WaveHoltz handles are RefWH (collocation) or RefWHQ (exact quadrature); the first
    // member records which
    struct WHHandle
    {
        bool exact;
        std::unique_ptr<RefWH> c;
        std::unique_ptr<RefWHQ> q;
    };
    template <class F>
    auto with_wh(void *w, F f)
    {
        WHHandle *h = static_cast<WHHandle *>(w);
        return h->exact ? f(*h->q) : f(*h->c);
    }
} // namespace

extern "C"
{
    void *ref_mesh_create(int nv, const double *xy, int nel, const int *quads)
    {
        return new RefMesh(Mesh2D::from_vertices(nv, xy, nel, quads));
    }
    // Mesh2D::from_file (source/Mesh2D.cpp:94-128), the reference's own reader; nullptr when it
    // reports an error
    void *ref_mesh_from_file(const char *dir)
    {
        try
        {
            return new RefMesh(Mesh2D::from_file(dir));
        }
        catch (const std::exception &)
        {
            return nullptr;
        }
    }
    void ref_mesh_destroy(void *m) { delete static_cast<RefMesh *>(m); }
    int ref_mesh_n_elem(void *m) { return static_cast<RefMesh *>(m)->mesh.n_elem(); }
    int ref_mesh_n_edges(void *m, int type) { return static_cast<RefMesh *>(m)->mesh.n_edges(face_type(type)); }
    double ref_mesh_min_h(void *m) { return static_cast<RefMesh *>(m)->mesh.min_h(); }

    // (el0, s0, el1, s1, delta) per edge of the given type, in the mesh's order
    void ref_mesh_edges(void *m, int type, int *out)
    {
        const Mesh2D &mesh = static_cast<RefMesh *>(m)->mesh;
        const FaceType ft = face_type(type);
        for (int e = 0; e < mesh.n_edges(ft); ++e)
        {
            const Edge *E = mesh.edge(e, ft);
            out[5 * e + 0] = E->elements[0];
            out[5 * e + 1] = E->sides[0];
            out[5 * e + 2] = (ft == FaceType::INTERIOR) ? E->elements[1] : -1;
            out[5 * e + 3] = (ft == FaceType::INTERIOR) ? E->sides[1] : -1;
            out[5 * e + 4] = (ft == FaceType::INTERIOR) ? E->delta : 1;
        }
    }

    // midpoint of every boundary edge (the examples' way of choosing codes)
    void ref_mesh_boundary_midpoints(void *m, double *xy)
    {
        const Mesh2D &mesh = static_cast<RefMesh *>(m)->mesh;
        auto q = QuadratureRule::quadrature_rule(1);
        const double *x = mesh.edge_metrics(q, FaceType::BOUNDARY).physical_coordinates();
        std::memcpy(xy, x, sizeof(double) * 2 * mesh.n_edges(FaceType::BOUNDARY));
    }

    void ref_basis(int n, double *x, double *w, double *D)
    {
        auto q = QuadratureRule::quadrature_rule(n, QuadratureRule::GaussLobatto);
        std::memcpy(x, q->x, sizeof(double) * n);
        std::memcpy(w, q->w, sizeof(double) * n);
        lagrange_basis_deriv(D, n, q->x, n, q->x);
    }

    void *ref_op_create(void *m, int n_colloc, const int *bc)
    {
        return new RefOp(static_cast<RefMesh *>(m)->mesh, n_colloc, bc);
    }
    void ref_op_destroy(void *o) { delete static_cast<RefOp *>(o); }

    void ref_node_coords(void *o, double *xy)
    {
        RefOp *op = static_cast<RefOp *>(o);
        const double *x = op->mesh.element_metrics(op->basis).physical_coordinates();
        std::memcpy(xy, x, sizeof(double) * 2 * op->n * op->n * op->nel);
    }

    void ref_div(void *o, const double *u, double *du) { static_cast<RefOp *>(o)->div().action(u, du); }
    void ref_wave_action(void *o, const double *u, double *du) { static_cast<RefOp *>(o)->a.action(u, du); }
    void ref_bc_action(void *o, const double *u, double *du) { static_cast<RefOp *>(o)->bc.action(u, du); }

    // the reference's WaveBC verbatim (codes 0/1 only); returns -1 when not
    // constructible.  Kept to document defect B1: two identical calls can
    // differ because absorb_2d reads state left over from the previous node.
    int ref_bc_action_native(void *o, const double *u, double *du)
    {
        RefOp *op = static_cast<RefOp *>(o);
        if (!op->native_bc)
            return -1;
        op->native_bc->action(u, du);
        return 0;
    }

    void ref_prolong(void *o, int type, const double *u, double *uf)
    {
        static_cast<RefOp *>(o)->prol(type).action(3, u, uf);
    }
    void ref_prolong_t(void *o, int type, const double *uf, double *u)
    {
        static_cast<RefOp *>(o)->prol(type).t(3, uf, u);
    }
    void ref_flux(void *o, int type, const double *uf, double *fb)
    {
        static_cast<RefOp *>(o)->flx(type).action(uf, fb);
    }
    void ref_apply_bc(void *o, double *uB) { static_cast<RefOp *>(o)->bc.exterior(uB); }
    void ref_mass_inv(void *o, int n_var, double *x) { static_cast<RefOp *>(o)->m.inv(n_var, x); }
    void ref_mass_action(void *o, int n_var, const double *x, double *y) { static_cast<RefOp *>(o)->m.action(n_var, x, y); }
    void ref_rhs(void *o, const double *u, double *du) { static_cast<RefOp *>(o)->rhs(u, du, nullptr, 0.0); }
    void ref_rhs_forced(void *o, const double *u, double *du, const double *F, double s)
    {
        static_cast<RefOp *>(o)->rhs(u, du, F, s);
    }

    // nsteps of the reference's low-storage RK4 (wavedg/ode.hpp:66-93) on
    // du/dt = M^{-1}(A + B) u
    void ref_rk4(void *o, double dt, int nsteps, double *t, double *u)
    {
        RefOp *op = static_cast<RefOp *>(o);
        ode::RungeKutta4 rk(op->ndof);
        auto f = [op](double *dudt, const double, const double *v)
        { op->rhs(v, dudt, nullptr, 0.0); };
        for (int s = 0; s < nsteps; ++s)
            rk.step(dt, f, *t, u);
    }

    // ---- Advection<true> ----
    void *ref_opa_create(void *m, int n_colloc, int nv, const double *a)
    {
        return new RefOpA(static_cast<RefMesh *>(m)->mesh, n_colloc, nv, a);
    }
    void ref_opa_destroy(void *o) { delete static_cast<RefOpA *>(o); }
    void ref_opa_action(void *o, const double *u, double *du) { static_cast<RefOpA *>(o)->adv.action(u, du); }
    void ref_opa_bc_action(void *o, const double *u, double *du) { static_cast<RefOpA *>(o)->bc.action(u, du); }
    void ref_opa_rhs(void *o, const double *u, double *du) { static_cast<RefOpA *>(o)->rhs(u, du); }
    void ref_opa_rk4(void *o, double dt, int nsteps, double *t, double *u)
    {
        RefOpA *op = static_cast<RefOpA *>(o);
        ode::RungeKutta4 rk(op->ndof);
        auto f = [op](double *dudt, const double, const double *v) { op->rhs(v, dudt); };
        for (int s = 0; s < nsteps; ++s)
            rk.step(dt, f, *t, u);
    }

    // ---- compressible Euler (examples/cl2d.cpp), DivF2D<true> / EdgeFluxF2D<true> ----
    void *ref_ope_create(void *m, int n_colloc) { return new RefOpE(static_cast<RefMesh *>(m)->mesh, n_colloc); }
    void ref_ope_destroy(void *o) { delete static_cast<RefOpE *>(o); }
    void ref_ope_div(void *o, const double *u, double *du)
    {
        static_cast<RefOpE *>(o)->div.action(RefOpE::nv, euler_flux, u, du);
    }
    void ref_ope_flux(void *o, int type, const double *ub, double *fb) { static_cast<RefOpE *>(o)->flux(type, ub, fb); }
    void ref_ope_prolong(void *o, int type, const double *u, double *ub)
    {
        RefOpE *op = static_cast<RefOpE *>(o);
        (type == 0 ? op->prolI : op->prolB)->action(RefOpE::nv, u, ub);
    }
    void ref_ope_rhs(void *o, const double *u, double *du) { static_cast<RefOpE *>(o)->rhs(u, du); }
    // method 0: ode::RungeKutta4, 1: ode::SSPRK3 (the stepper examples/cl2d.cpp uses)
    void ref_ope_steps(void *o, int method, double dt, int nsteps, double *t, double *u)
    {
        RefOpE *op = static_cast<RefOpE *>(o);
        auto f = [op](double *dudt, const double, const double *v) { op->rhs(v, dudt); };
        if (method == 0)
        {
            ode::RungeKutta4 rk(op->ndof);
            for (int s = 0; s < nsteps; ++s)
                rk.step(dt, f, *t, u);
        }
        else
        {
            ode::SSPRK3 rk(op->ndof);
            for (int s = 0; s < nsteps; ++s)
                rk.step(dt, f, *t, u);
        }
    }

    // ---- Advection with a spatially varying coefficient ----
    // basis_type: 0 Gauss-Legendre, 1 Gauss-Lobatto (QuadratureRule::QuadratureType's order)
    void *ref_opv_create(void *m, int n_colloc, int nv, const double *a, int approx, int basis_type)
    {
        const Mesh2D &mesh = static_cast<RefMesh *>(m)->mesh;
        const auto type = basis_type == 0 ? QuadratureRule::GaussLegendre : QuadratureRule::GaussLobatto;
        if (approx)
            return static_cast<RefOpVBase *>(new RefOpV<true>(mesh, n_colloc, nv, a, type));
        return static_cast<RefOpVBase *>(new RefOpV<false>(mesh, n_colloc, nv, a, type));
    }
    void ref_opv_destroy(void *o) { delete static_cast<RefOpVBase *>(o); }
    void ref_opv_action(void *o, const double *u, double *du) { static_cast<RefOpVBase *>(o)->action(u, du); }
    void ref_opv_bc_action(void *o, const double *u, double *du) { static_cast<RefOpVBase *>(o)->bc_action(u, du); }
    void ref_opv_rhs(void *o, const double *u, double *du) { static_cast<RefOpVBase *>(o)->rhs(u, du); }
    void ref_opv_steps(void *o, int method, double dt, int nsteps, double *t, double *u)
    {
        RefOpVBase *op = static_cast<RefOpVBase *>(o);
        auto f = [op](double *dudt, const double, const double *v) { op->rhs(v, dudt); };
        if (method == 0)
        {
            ode::RungeKutta4 rk(op->ndof);
            for (int s = 0; s < nsteps; ++s)
                rk.step(dt, f, *t, u);
        }
        else
        {
            ode::SSPRK3 rk(op->ndof);
            for (int s = 0; s < nsteps; ++s)
                rk.step(dt, f, *t, u);
        }
    }

    // ---- MassMatrix<AQ> and LinearFunctional2D on a basis of either type ----
    struct RefMassB
    {
        const QuadratureRule *basis;
        bool approx;
        std::unique_ptr<MassMatrix<true>> mt;
        std::unique_ptr<MassMatrix<false>> mf;
        LinearFunctional2D lf;
        int nel;
        RefMassB(const Mesh2D &mesh, int n, QuadratureRule::QuadratureType type, bool approx_)
            : basis(QuadratureRule::quadrature_rule(n, type)), approx(approx_), lf(mesh, basis), nel(mesh.n_elem())
        {
            if (approx)
                mt = std::make_unique<MassMatrix<true>>(mesh, basis);
            else
                mf = std::make_unique<MassMatrix<false>>(mesh, basis);
        }
    };
    // basis_type: 0 Gauss-Legendre, 1 Gauss-Lobatto
    void *ref_mb_create(void *m, int n_colloc, int basis_type, int approx)
    {
        return new RefMassB(static_cast<RefMesh *>(m)->mesh, n_colloc,
                            basis_type == 0 ? QuadratureRule::GaussLegendre : QuadratureRule::GaussLobatto, approx != 0);
    }
    void ref_mb_destroy(void *o) { delete static_cast<RefMassB *>(o); }
    void ref_mb_action(void *o, int nv, const double *x, double *y)
    {
        RefMassB *b = static_cast<RefMassB *>(o);
        if (b->approx)
            b->mt->action(nv, x, y);
        else
            b->mf->action(nv, x, y);
    }
    void ref_mb_inv(void *o, int nv, double *x)
    {
        RefMassB *b = static_cast<RefMassB *>(o);
        if (b->approx)
            b->mt->inv(nv, x);
        else
            b->mf->inv(nv, x);
    }
    // the points at which LinearFunctional2D::action evaluates f, in its call order
    // (x, y per point; point k + n (l + n el) of its default n-point rule)
    void ref_mb_points(void *o, double *xy)
    {
        RefMassB *b = static_cast<RefMassB *>(o);
        long long p = 0;
        std::vector<double> F((size_t)b->basis->n * b->basis->n * b->nel);
        auto f = [&](const double *x, double *out)
        {
            xy[2 * p] = x[0];
            xy[2 * p + 1] = x[1];
            ++p;
            out[0] = 0.0;
        };
        b->lf.action(1, f, F.data());
    }
    // LinearFunctional2D::action with f given by its values fq(d, point) at those points
    void ref_mb_load(void *o, int nv, const double *fq, double *F)
    {
        RefMassB *b = static_cast<RefMassB *>(o);
        long long p = 0;
        auto f = [&](const double *, double *out)
        {
            for (int d = 0; d < nv; ++d)
                out[d] = fq[(size_t)nv * p + d];
            ++p;
        };
        b->lf.action(nv, f, F);
    }

    // ---- compressible Euler with approx_quad = false (examples/cl2d.cpp as shipped) ----
    void *ref_opeq_create(void *m, int n_colloc) { return new RefOpEQ(static_cast<RefMesh *>(m)->mesh, n_colloc); }
    void ref_opeq_destroy(void *o) { delete static_cast<RefOpEQ *>(o); }
    void ref_opeq_div(void *o, const double *u, double *du)
    {
        static_cast<RefOpEQ *>(o)->div.action(RefOpEQ::nv, euler_flux, u, du);
    }
    void ref_opeq_flux(void *o, int type, const double *ub, double *fb) { static_cast<RefOpEQ *>(o)->flux(type, ub, fb); }
    void ref_opeq_rhs(void *o, const double *u, double *du) { static_cast<RefOpEQ *>(o)->rhs(u, du); }
    void ref_opeq_steps(void *o, int method, double dt, int nsteps, double *t, double *u)
    {
        RefOpEQ *op = static_cast<RefOpEQ *>(o);
        auto f = [op](double *dudt, const double, const double *v) { op->rhs(v, dudt); };
        if (method == 0)
        {
            ode::RungeKutta4 rk(op->ndof);
            for (int s = 0; s < nsteps; ++s)
                rk.step(dt, f, *t, u);
        }
        else
        {
            ode::SSPRK3 rk(op->ndof);
            for (int s = 0; s < nsteps; ++s)
                rk.step(dt, f, *t, u);
        }
    }

    // ---- exact quadrature (approx_quad = false) ----
    void *ref_opq_create(void *m, int n_colloc, const int *bc)
    {
        return new RefOpQ(static_cast<RefMesh *>(m)->mesh, n_colloc, bc);
    }
    void ref_opq_destroy(void *o) { delete static_cast<RefOpQ *>(o); }
    void ref_opq_div(void *o, const double *u, double *du) { static_cast<RefOpQ *>(o)->div.action(u, du); }
    void ref_opq_flux(void *o, int type, const double *uf, double *fb)
    {
        RefOpQ *op = static_cast<RefOpQ *>(o);
        (type == 0 ? op->flxI : op->flxB).action(uf, fb);
    }
    void ref_opq_wave_action(void *o, const double *u, double *du) { static_cast<RefOpQ *>(o)->a.action(u, du); }
    void ref_opq_bc_action(void *o, const double *u, double *du) { static_cast<RefOpQ *>(o)->bc.action(u, du); }
    void ref_opq_mass_inv(void *o, int n_var, double *x) { static_cast<RefOpQ *>(o)->m.inv(n_var, x); }
    void ref_opq_mass_action(void *o, int n_var, const double *x, double *y)
    {
        static_cast<RefOpQ *>(o)->m.action(n_var, x, y);
    }
    void ref_opq_rhs(void *o, const double *u, double *du) { static_cast<RefOpQ *>(o)->rhs(u, du); }
    void ref_opq_rk4(void *o, double dt, int nsteps, double *t, double *u)
    {
        RefOpQ *op = static_cast<RefOpQ *>(o);
        ode::RungeKutta4 rk(op->ndof);
        auto f = [op](double *dudt, const double, const double *v) { op->rhs(v, dudt); };
        for (int s = 0; s < nsteps; ++s)
            rk.step(dt, f, *t, u);
    }

    // (f, phi) with the reference's LinearFunctional2D for the field
    //   f_c(x) = scale * sum_k amp_k exp(-|x - c_k|^2 / (2 sigma_k^2)),
    // placed in component `comp` (other components 0).  With mass_inv != 0 the
    // result is M^{-1} (f, phi) (how the examples build initial states).
    void ref_load_gaussians(void *o, int nsrc, const double *cx, const double *cy, const double *sigma,
                            const double *amp, double scale, int comp, int mass_inv, double *F)
    {
        RefOp *op = static_cast<RefOp *>(o);
        LinearFunctional2D L(op->mesh, op->basis);
        auto f = [=](const double *x, double *out)
        {
            double s = 0.0;
            for (int k = 0; k < nsrc; ++k)
            {
                const double dx = x[0] - cx[k], dy = x[1] - cy[k];
                s += amp[k] * std::exp(-(dx * dx + dy * dy) / (2.0 * sigma[k] * sigma[k]));
            }
            out[0] = out[1] = out[2] = 0.0;
            out[comp] = scale * s;
        };
        L.action(3, f, F);
        if (mass_inv)
            op->m.inv(3, F);
    }

    double ref_norm(int n, const double *x) { return norm(n, x); }
    double ref_error(int n, const double *x, const double *y) { return error(n, x, y); }

    void *ref_wh_create(void *o, double omega)
    {
        return new WHHandle{false, std::make_unique<RefWH>(*static_cast<RefOp *>(o), omega), nullptr};
    }
    void *ref_whq_create(void *o, double omega)
    {
        return new WHHandle{true, nullptr, std::make_unique<RefWHQ>(*static_cast<RefOpQ *>(o), omega)};
    }
    void ref_wh_destroy(void *w) { delete static_cast<WHHandle *>(w); }
    void ref_wh_params(void *w, double *T, double *dt, int *nt)
    {
        with_wh(w, [&](auto &wh) { *T = wh.T; *dt = wh.dt; *nt = wh.nt; return 0; });
    }
    int ref_wh_is_native(void *w) { return with_wh(w, [](auto &wh) { return wh.native ? 1 : 0; }); }
    void ref_wh_pi0(void *w, double *u, const double *F) { with_wh(w, [&](auto &wh) { wh.pi0(u, F); return 0; }); }
    void ref_wh_S(void *w, double *u) { with_wh(w, [&](auto &wh) { wh.S(u); return 0; }); }
    void ref_wh_postprocess(void *w, double *H, const double *U)
    {
        with_wh(w, [&](auto &wh) { wh.postprocess(H, U); return 0; });
    }

    // the fixed-point loop of examples/waveholtz2d.cpp:165-185 from W (in/out)
    int ref_wh_solve(void *w, const double *pi0, double tol, int maxit, double *W, double *err_out)
    {
        const int ndof = with_wh(w, [](auto &wh) { return wh.op.ndof; });
        const double pz = norm(ndof, pi0);
        std::vector<double> prev(ndof);
        int it;
        double err = 0.0;
        for (it = 1; it <= maxit; ++it)
        {
            std::memcpy(prev.data(), W, sizeof(double) * ndof);
            ref_wh_S(w, W);
            for (int i = 0; i < ndof; ++i)
                W[i] += pi0[i];
            err = error(ndof, W, prev.data()) / pz;
            if (err < tol)
                break;
        }
        *err_out = err;
        return it;
    }
}
