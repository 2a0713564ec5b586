// wdg_b200.hpp -- drop-in C++ classes for the reference waveDG interface.
//
// Include after the reference's headers (its include directories and the
// generated wdg_config.hpp on the include path).  Each class derives from the
// reference's own dg::Operator / dg::InvertibleOperator and takes the same
// constructor arguments as the reference class it replaces, so a driver only
// changes type names (dg::WaveEquation -> dg::b200::WaveEquation, ...).  All work
// happens on the GPU through the C ABI in wdg_b200.h; host arrays are staged,
// device arrays are used in place.  Errors throw std::runtime_error, like the
// reference's wdg_error (source/wdg_error.cpp:5-20).
#ifndef WDG_B200_HPP
#define WDG_B200_HPP

#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "wdg_b200.h"

namespace dg
{
namespace b200
{
    inline void check(int status)
    {
        if (status < 0)
            throw std::runtime_error(std::string("wdg_b200: ") + wdg_last_error());
    }

    // A dg::Mesh2D adopted through its public API: corners from QuadElement::corner
    // (wavedg/Element.hpp:123-126) and the edge tables in Mesh2D::edge(i, type) order.
    class Mesh
    {
    public:
        explicit Mesh(const dg::Mesh2D &m)
        {
            const int nel = m.n_elem();
            std::vector<double> corners(8 * (size_t)nel);
            for (int el = 0; el < nel; ++el)
            {
                const auto *q = dynamic_cast<const dg::QuadElement *>(m.element(el));
                if (!q)
                    throw std::runtime_error("wdg_b200: only QuadElement meshes are supported");
                for (int c = 0; c < 4; ++c)
                {
                    corners[8 * (size_t)el + 2 * c] = q->corner(c)[0];
                    corners[8 * (size_t)el + 2 * c + 1] = q->corner(c)[1];
                }
            }
            auto table = [&](dg::FaceType t)
            {
                std::vector<int> out(5 * (size_t)m.n_edges(t));
                for (int e = 0; e < m.n_edges(t); ++e)
                {
                    const dg::Edge *E = m.edge(e, t);
                    out[5 * e] = E->elements[0];
                    out[5 * e + 1] = E->sides[0];
                    out[5 * e + 2] = (t == dg::FaceType::INTERIOR) ? E->elements[1] : -1;
                    out[5 * e + 3] = (t == dg::FaceType::INTERIOR) ? E->sides[1] : -1;
                    out[5 * e + 4] = (t == dg::FaceType::INTERIOR) ? E->delta : 1;
                }
                return out;
            };
            const std::vector<int> ie = table(dg::FaceType::INTERIOR), be = table(dg::FaceType::BOUNDARY);
            wdg_mesh *h = nullptr;
            check(wdg_mesh_from_tables(nel, corners.data(), (int)(ie.size() / 5), ie.data(), (int)(be.size() / 5),
                                       be.data(), &h));
            h_.reset(h, wdg_mesh_destroy);
        }
        wdg_mesh *get() const { return h_.get(); }
        int n_boundary() const { return wdg_mesh_n_edges(h_.get(), WDG_BOUNDARY); }

    private:
        std::shared_ptr<wdg_mesh> h_;
    };

    // one GPU discretisation of the wave system (geometry on the device)
    class Discretisation
    {
    public:
        Discretisation(const dg::Mesh2D &mesh, const dg::QuadratureRule *basis, const int *bc, int precision = WDG_FP64,
                       int device = -1)
            : mesh_(mesh)
        {
            if (!basis || basis->type != dg::QuadratureRule::GaussLobatto)
                throw std::runtime_error("wdg_b200: the GPU operators are built for Gauss-Lobatto bases");
            wdg_wave *w = nullptr;
            check(wdg_wave_create(mesh_.get(), basis->n, bc, precision, device, &w));
            h_.reset(w, wdg_wave_destroy);
            long long nd = 0;
            check(wdg_wave_info(w, nullptr, nullptr, &nd, nullptr));
            ndof_ = nd;
        }
        wdg_wave *get() const { return h_.get(); }
        long long ndof() const { return ndof_; }

    private:
        Mesh mesh_;
        std::shared_ptr<wdg_wave> h_;
        long long ndof_ = 0;
    };

    inline void require_approx(bool approx_quad)
    {
        if (!approx_quad)
            throw std::runtime_error("wdg_b200: this class is built for approx_quad = true");
    }

    // the same system with approx_quad = false: Div<false>, EdgeFlux<false>, MassMatrix<false>
    // with the reference's default quadrature rules (FP64)
    class ExactDiscretisation
    {
    public:
        ExactDiscretisation(const dg::Mesh2D &mesh, const dg::QuadratureRule *basis, const int *bc,
                            const dg::QuadratureRule *quad = nullptr, int device = -1)
            : mesh_(mesh)
        {
            if (!basis || basis->type != dg::QuadratureRule::GaussLobatto)
                throw std::runtime_error("wdg_b200: the GPU operators are built for Gauss-Lobatto bases");
            if (quad)
                throw std::runtime_error("wdg_b200: exact quadrature is built for the default rules (quad = nullptr)");
            wdg_waveq *q = nullptr;
            check(wdg_waveq_create(mesh_.get(), basis->n, bc, device, &q));
            h_.reset(q, wdg_waveq_destroy);
        }
        wdg_waveq *get() const { return h_.get(); }

    private:
        Mesh mesh_;
        std::shared_ptr<wdg_waveq> h_;
    };

    // dg::WaveEquation (source/WaveEquation.cpp:5-68): du += Div(u) + P^T Flux(P u)
    class WaveEquation : public dg::Operator
    {
    public:
        WaveEquation(const dg::Mesh2D &mesh, const dg::QuadratureRule *basis, bool approx_quad = false,
                     const dg::QuadratureRule *quad = nullptr)
        {
            if (approx_quad)
                d_ = std::make_shared<Discretisation>(mesh, basis, nullptr);
            else
                q_ = std::make_shared<ExactDiscretisation>(mesh, basis, nullptr, quad);
        }
        void action(const double *u, double *du) const override
        {
            check(d_ ? wdg_wave_action(d_->get(), u, du) : wdg_waveq_wave_action(q_->get(), u, du));
        }
        void action(int, const double *u, double *du) const override { action(u, du); }

    private:
        std::shared_ptr<Discretisation> d_;
        std::shared_ptr<ExactDiscretisation> q_;
    };

    // dg::WaveBC (source/WaveEquation.cpp:70-215); codes 0 absorbing, 1 reflecting, 2 Dirichlet p = 0
    class WaveBC : public dg::Operator
    {
    public:
        WaveBC(const dg::Mesh2D &mesh, const int *bc, const dg::QuadratureRule *basis, bool approx_quad,
               const dg::QuadratureRule *quad = nullptr)
        {
            if (approx_quad)
                d_ = std::make_shared<Discretisation>(mesh, basis, bc);
            else
                q_ = std::make_shared<ExactDiscretisation>(mesh, basis, bc, quad);
        }
        void action(const double *u, double *du) const override
        {
            check(d_ ? wdg_wavebc_action(d_->get(), u, du) : wdg_waveq_wavebc_action(q_->get(), u, du));
        }
        void action(int, const double *u, double *du) const override { action(u, du); }

    private:
        std::shared_ptr<Discretisation> d_;
        std::shared_ptr<ExactDiscretisation> q_;
    };

    // dg::MassMatrix<true> (source/MassMatrix.cpp:6-82) and, APPROX = false, MassMatrix<false>
    // (block Cholesky of the exact element mass matrices, :84-230)
    template <bool APPROX = true>
    class MassMatrix : public dg::InvertibleOperator
    {
    public:
        MassMatrix(const dg::Mesh2D &mesh, const dg::QuadratureRule *basis, const dg::QuadratureRule *quad = nullptr)
        {
            if (APPROX)
                d_ = std::make_shared<Discretisation>(mesh, basis, nullptr);
            else
                q_ = std::make_shared<ExactDiscretisation>(mesh, basis, nullptr, quad);
        }
        void action(const double *x, double *y) const override { action(1, x, y); }
        void action(int n_var, const double *x, double *y) const override
        {
            check(d_ ? wdg_mass_action(d_->get(), n_var, x, y) : wdg_waveq_mass_action(q_->get(), n_var, x, y));
        }
        void inv(double *x) const override { inv(1, x); }
        void inv(int n_var, double *x) const override
        {
            check(d_ ? wdg_mass_inv(d_->get(), n_var, x) : wdg_waveq_mass_inv(q_->get(), n_var, x));
        }

    private:
        std::shared_ptr<Discretisation> d_;
        std::shared_ptr<ExactDiscretisation> q_;
    };

    // The examples' time derivative M^{-1}(A + B) u as one fused operator, with the
    // fused ode::RungeKutta4 (wavedg/ode.hpp:66-93) stepping on the GPU.
    class WaveSystem : public dg::Operator
    {
    public:
        WaveSystem(const dg::Mesh2D &mesh, const dg::QuadratureRule *basis, const int *bc, int precision = WDG_FP64)
            : d_(mesh, basis, bc, precision) {}
        // y <- M^{-1} (A + B) x  (overwrites y)
        void action(const double *x, double *y) const override { check(wdg_rhs(d_.get(), x, y, nullptr, 0.0)); }
        void action(int, const double *x, double *y) const override { action(x, y); }
        // ode::RungeKutta4::step, `nsteps` times: t += nsteps * dt, u in place
        void rk4_steps(double dt, double &t, double *u, int nsteps = 1) const
        {
            check(wdg_rk4_steps(d_.get(), u, dt, &t, nsteps));
        }
        void autotune(int steps = 5) const { check(wdg_wave_autotune(d_.get(), steps, nullptr)); }
        wdg_wave *get() const { return d_.get(); }
        long long ndof() const { return d_.ndof(); }

    private:
        Discretisation d_;
    };

    // dg::WaveHoltz (source/WaveHoltz.cpp)
    class WaveHoltz
    {
    public:
        WaveHoltz(double omega, const dg::Mesh2D &mesh, const dg::QuadratureRule *basis, const int *bc,
                  bool approx_quad = false, int precision = WDG_FP64)
            : omega_(omega)
        {
            wdg_waveholtz *h = nullptr;
            if (approx_quad)
            {
                sys_ = std::make_shared<WaveSystem>(mesh, basis, bc, precision);
                check(wdg_waveholtz_create(sys_->get(), omega, &h));
            }
            else
            {
                if (precision != WDG_FP64)
                    throw std::runtime_error("wdg_b200: exact-quadrature WaveHoltz is FP64");
                q_ = std::make_shared<ExactDiscretisation>(mesh, basis, bc);
                check(wdg_waveholtz_create_exact(q_->get(), omega, &h));
            }
            h_.reset(h, wdg_waveholtz_destroy);
        }
        double K(double t) const { return omega_ / M_PI * (std::cos(omega_ * t) - 0.25); }
        void pi0(double *w, const double *F) const { check(wdg_waveholtz_pi0(h_.get(), w, F)); }
        void S(double *w) const { check(wdg_waveholtz_S(h_.get(), w)); }
        void postprocess(double *H, const double *w) const { check(wdg_waveholtz_postprocess(h_.get(), H, w)); }
        // the fixed-point loop of examples/waveholtz2d.cpp:137-185; returns the iterations taken
        int solve(const double *F, double tol, int maxit, double *W, double *residual) const
        {
            int it = 0;
            const int s = wdg_waveholtz_solve(h_.get(), F, tol, maxit, W, &it, residual);
            if (s != WDG_ERR_NOT_CONVERGED)
                check(s);
            return it;
        }

    private:
        double omega_;
        std::shared_ptr<WaveSystem> sys_;
        std::shared_ptr<ExactDiscretisation> q_;
        std::shared_ptr<wdg_waveholtz> h_; // released first (declared last)
    };

    // Many independent WaveHoltz solves advanced together (wdg_whbatch_*; no reference
    // counterpart: the reference runs one WaveHoltz object at a time).  The systems must share
    // one precision and device and outlive the batch.
    class WaveHoltzBatch
    {
    public:
        struct Result
        {
            std::vector<int> iterations, status; // status 0 converged, 1 maxit, 2 stalled
            std::vector<double> residual, pi0_norm;
        };
        WaveHoltzBatch(const std::vector<const WaveSystem *> &systems, const std::vector<double> &omegas)
            : n_((int)systems.size())
        {
            if (omegas.size() != systems.size())
                throw std::runtime_error("wdg_b200: one frequency per solve");
            std::vector<wdg_wave *> w;
            for (const WaveSystem *s : systems)
                w.push_back(s->get());
            wdg_whbatch *h = nullptr;
            check(wdg_whbatch_create(n_, w.data(), omegas.data(), &h));
            h_.reset(h, wdg_whbatch_destroy);
        }
        float autotune(int steps = 64) const
        {
            float ms = 0.f;
            check(wdg_whbatch_autotune(h_.get(), steps, &ms));
            return ms;
        }
        // F[s], W[s]: FP64 arrays of solve s (host or device); W receives the iterates.
        // warm (optional): per solve, start from W[s]; pi0_norm (optional): known |pi0| per solve
        Result solve(const std::vector<const double *> &F, const std::vector<double *> &W, double tol, int maxit,
                     int stall_limit = 0, const std::vector<int> &warm = {},
                     const std::vector<double> &pi0_norm = {}) const
        {
            if ((int)F.size() != n_ || (int)W.size() != n_ || (!warm.empty() && (int)warm.size() != n_) ||
                (!pi0_norm.empty() && (int)pi0_norm.size() != n_))
                throw std::runtime_error("wdg_b200: one forcing, iterate (and flag) per solve");
            Result r;
            r.iterations.assign(n_, 0);
            r.status.assign(n_, -1);
            r.residual.assign(n_, 0.0);
            r.pi0_norm = pi0_norm.empty() ? std::vector<double>(n_, 0.0) : pi0_norm;
            check(wdg_whbatch_solve(h_.get(), F.data(), tol, maxit, stall_limit, W.data(),
                                    warm.empty() ? nullptr : warm.data(), r.pi0_norm.data(), r.iterations.data(),
                                    r.residual.data(), r.status.data()));
            return r;
        }

    private:
        int n_;
        std::shared_ptr<wdg_whbatch> h_;
    };

    // The compressible Euler system of examples/cl2d.cpp (DivF2D, EdgeFluxF2D with the example's
    // flux and local Lax-Friedrichs numerical flux, exterior boundary state = interior state,
    // MassMatrix) as one fused operator, with the example's approx_quad switch as a template
    // argument (false, the example's setting: 2n-point Gauss-Legendre rules and the dense
    // inverse mass matrix): action(u, dudt) overwrites dudt with the example's time derivative.
    // The flux model is built into the kernels (a GPU kernel needs its flux at compile time).
    template <bool ApproxQuad = true>
    class EulerSystem : public dg::Operator
    {
    public:
        EulerSystem(const dg::Mesh2D &mesh, const dg::QuadratureRule *basis, int device = -1)
        {
            if (basis->type != dg::QuadratureRule::GaussLobatto)
                throw std::runtime_error("wdg_b200: the Euler kernels are built for Gauss-Lobatto bases");
            Mesh m(mesh);
            wdg_claw *h = nullptr;
            check(ApproxQuad ? wdg_euler_create(m.get(), basis->n, device, &h)
                             : wdg_euler_create_exact(m.get(), basis->n, device, &h));
            h_.reset(h, wdg_claw_destroy);
        }
        void action(const double *u, double *dudt) const override { check(wdg_claw_rhs(h_.get(), u, dudt)); }
        void action(int, const double *u, double *dudt) const override { action(u, dudt); }
        // DivF2D<ApproxQuad>::action: divF += (F(u), grad v)
        void div(const double *u, double *divF) const { check(wdg_claw_div(h_.get(), u, divF)); }
        // ode::SSPRK3::step (the example's stepper) or, with rk4, ode::RungeKutta4::step, nsteps times
        void steps(double dt, double &t, double *u, int nsteps = 1, bool rk4 = false) const
        {
            check(wdg_claw_steps(h_.get(), rk4 ? 0 : 1, u, dt, &t, nsteps));
        }

    private:
        std::shared_ptr<wdg_claw> h_;
    };

    // Linear advection (wavedg/Advection.hpp:17-273) on the GPU for any coefficient, basis and
    // quadrature of the reference's Advection<ApproxQuad>: a spatially varying coefficient
    // a(n_var, n_var, 2, n, n, n_elem), or a constant one (n_var, n_var, 2) spread to the
    // nodes.  n.A must be scalar or symmetric.  The handle behind these classes holds the
    // operator tables the reference builds at construction.
    inline std::shared_ptr<wdg_vadvect> make_advection(int n_var, const dg::Mesh2D &mesh, const dg::QuadratureRule *basis,
                                                       const double *a, bool constant_coefficient, bool approx_quad,
                                                       int device)
    {
        const int n = basis->n, nel = mesh.n_elem(), per = 2 * n_var * n_var;
        std::vector<double> spread;
        if (constant_coefficient)
        {
            spread.resize((size_t)per * n * n * nel);
            for (size_t p = 0; p < (size_t)n * n * nel; ++p)
                for (int k = 0; k < per; ++k)
                    spread[(size_t)per * p + k] = a[k];
            a = spread.data();
        }
        const int type = basis->type == dg::QuadratureRule::GaussLegendre ? WDG_GAUSS_LEGENDRE : WDG_GAUSS_LOBATTO;
        Mesh m(mesh);
        wdg_vadvect *h = nullptr;
        check(wdg_vadvect_create(m.get(), n, type, n_var, a, approx_quad ? 1 : 0, device, &h));
        return std::shared_ptr<wdg_vadvect>(h, wdg_vadvect_destroy);
    }

    template <bool ApproxQuad>
    class Advection : public dg::Operator
    {
    public:
        Advection(int n_var, const dg::Mesh2D &mesh, const dg::QuadratureRule *basis, const double *a,
                  bool constant_coefficient, int device = -1)
            : h_(make_advection(n_var, mesh, basis, a, constant_coefficient, ApproxQuad, device))
        {
        }
        // du += (A u, grad v) - interior fluxes
        void action(const double *u, double *du) const override { check(wdg_vadvect_action(h_.get(), u, du)); }
        void action(int, const double *u, double *du) const override { action(u, du); }

    private:
        std::shared_ptr<wdg_vadvect> h_;
    };

    template <bool ApproxQuad>
    class AdvectionHomogeneousBC : public dg::Operator
    {
    public:
        AdvectionHomogeneousBC(int n_var, const dg::Mesh2D &mesh, const dg::QuadratureRule *basis, const double *a,
                               bool constant_coefficient, int device = -1)
            : h_(make_advection(n_var, mesh, basis, a, constant_coefficient, ApproxQuad, device))
        {
        }
        // du += boundary fluxes with u = 0 outside the domain
        void action(const double *u, double *du) const override { check(wdg_vadvect_bc_action(h_.get(), u, du)); }
        void action(int, const double *u, double *du) const override { action(u, du); }

    private:
        std::shared_ptr<wdg_vadvect> h_;
    };

    // The time derivative of examples/advec2d.cpp as one operator: action(u, dudt) overwrites
    // dudt with M^{-1} (Advection + AdvectionHomogeneousBC) u; steps() runs ode::SSPRK3 (the
    // example's stepper) or ode::RungeKutta4 with one fused launch per stage.
    template <bool ApproxQuad>
    class AdvectionSystem : public dg::Operator
    {
    public:
        AdvectionSystem(int n_var, const dg::Mesh2D &mesh, const dg::QuadratureRule *basis, const double *a,
                        bool constant_coefficient, int device = -1)
            : h_(make_advection(n_var, mesh, basis, a, constant_coefficient, ApproxQuad, device))
        {
        }
        void action(const double *u, double *dudt) const override { check(wdg_vadvect_rhs(h_.get(), u, dudt)); }
        void action(int, const double *u, double *dudt) const override { action(u, dudt); }
        void steps(double dt, double &t, double *u, int nsteps = 1, bool rk4 = false) const
        {
            check(wdg_vadvect_steps(h_.get(), rk4 ? 0 : 1, u, dt, &t, nsteps));
        }

    private:
        std::shared_ptr<wdg_vadvect> h_;
    };
} // namespace b200
} // namespace dg

#endif
